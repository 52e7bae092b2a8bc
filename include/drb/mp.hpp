// drb/mp.hpp -- C++ host mirror of the reference's dr::mp gemv interface,
// header-only over the C ABI of drb.h (no CUDA headers needed to include it).
//
// Mirrors (paths relative to the reference project):
//   drb::index, drb::matrix_entry          include/dr/detail/index.hpp,
//                                          include/dr/detail/matrix_entry.hpp
//   drb::views::csr_matrix_view            include/dr/views/csr_matrix_view.hpp:125-220
//   drb::generate_random_csr / _band_csr   include/dr/detail/generate_csr.hpp:40-153
//   drb::mp::distribution                  include/dr/mp/containers/distribution.hpp:11-44
//   drb::mp::csr_row_distribution          .../matrix_formats/csr_row_distribution.hpp
//   drb::mp::csr_eq_distribution           .../matrix_formats/csr_eq_distribution.hpp
//   drb::mp::distributed_sparse_matrix     .../distributed_sparse_matrix.hpp:29-162
//   drb::mp::broadcasted_vector            .../broadcasted_vector.hpp:9-51
//   drb::mp::broadcasted_slim_matrix       .../broadcasted_slim_matrix.hpp:9-80
//   drb::mp::gemv (4 overloads)            include/dr/mp/algorithms/matrix/gemv.hpp:16-71
//   drb::mp::distributed_vector            .../distributed_vector.hpp:150-340
//   drb::mp::reduce (range and iterator    include/dr/mp/algorithms/reduce.hpp:127-232
//     overloads), iota, fill               .../iota.hpp:20-34, .../fill.hpp:21-30
//   drb::mp::conjugate_gradient            no reference counterpart (drb_csr_cg)
//
// Differences that follow from "one process owns one GPU":
//   * default_comm() is rank 0 of 1; every segment of a matrix lives on the
//     current GPU and one kernel launch covers all of them;
//   * broadcasted_* data lives in device memory; operator[] returns a copy;
//   * failures throw drb::error (the reference asserts); the C ABI itself
//     never throws.
#pragma once

#include <algorithm>
#include <cassert>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <iterator>
#include <random>
#include <ranges>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../drb.h"

namespace drb {

struct error : std::runtime_error {
  drb_status status;
  error(drb_status s, const std::string &msg)
      : std::runtime_error(msg), status(s) {}
};

inline void check(drb_status s) {
  if (s != DRB_OK)
    throw error(s, std::string("drb: ") + drb_last_error());
}

// ---- index / matrix_entry ---------------------------------------------------
template <std::integral T = std::size_t> struct index {
  using index_type = T;
  T first = 0, second = 0;
  constexpr index() = default;
  constexpr index(T a, T b) : first(a), second(b) {}
  constexpr T operator[](T dim) const { return dim == 0 ? first : second; }
  template <std::size_t N> constexpr T get() const {
    return N == 0 ? first : second;
  }
  constexpr bool operator==(const index &) const = default;
};

template <typename T, std::integral I = std::size_t> struct matrix_entry {
  using index_type = I;
  using value_type = T;
  index<I> idx;
  T val;
  matrix_entry() = default;
  matrix_entry(index<I> i, T v) : idx(i), val(v) {}
  index<I> index_() const { return idx; }
  T value() const { return val; }
  template <std::size_t N> decltype(auto) get() const {
    if constexpr (N == 0)
      return idx;
    else
      return val;
  }
  bool operator==(const matrix_entry &) const = default;
};

namespace detail {
template <class T> constexpr drb_dtype dtype_of() {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>,
                "element type must be float or double");
  return std::is_same_v<T, float> ? DRB_F32 : DRB_F64;
}
template <class I> constexpr drb_itype itype_of() {
  static_assert(std::is_integral_v<I> && (sizeof(I) == 4 || sizeof(I) == 8),
                "index type must be a 32- or 64-bit integer");
  return sizeof(I) == 8 ? DRB_I64 : DRB_I32;
}
} // namespace detail

namespace views {

// Non-owning CSR triple on the host (csr_matrix_view.hpp:125-220).
template <typename T, typename I, typename TIter = T *, typename IIter = I *>
class csr_matrix_view {
public:
  using scalar_type = T;
  using index_type = I;
  using key_type = drb::index<I>;
  using size_type = std::size_t;

  csr_matrix_view() = default;
  csr_matrix_view(TIter values, IIter rowptr, IIter colind, key_type shape,
                  size_type nnz, size_type rank)
      : values_(values), rowptr_(rowptr), colind_(colind), shape_(shape),
        nnz_(nnz), rank_(rank) {}

  key_type shape() const noexcept { return shape_; }
  size_type size() const noexcept { return nnz_; }
  size_type rank() const { return rank_; }
  TIter values_data() const { return values_; }
  IIter rowptr_data() const { return rowptr_; }
  IIter colind_data() const { return colind_; }

  // Entries in CSR order as matrix_entry values.
  std::vector<matrix_entry<T, I>> entries() const {
    std::vector<matrix_entry<T, I>> out;
    out.reserve(nnz_);
    for (I r = 0; r < shape_[0]; r++)
      for (auto p = rowptr_[r]; p < rowptr_[r + 1]; p++)
        out.emplace_back(key_type(r, colind_[p]), values_[p]);
    return out;
  }

private:
  TIter values_{};
  IIter rowptr_{};
  IIter colind_{};
  key_type shape_{};
  size_type nnz_ = 0;
  size_type rank_ = 0;
};

} // namespace views

// ---- generators (generate_csr.hpp:40-153) ------------------------------------
// Same engine, distributions, draw order and CSR fill as the reference, so a
// given (shape, density, seed) yields the same matrix under libstdc++.
template <typename T = float, std::integral I = std::size_t>
auto generate_random_csr(index<I> shape, double density = 0.01,
                         unsigned int seed = 0) {
  assert(density >= 0.0 && density < 1.0);
  struct hash {
    std::size_t operator()(const std::pair<I, I> &v) const {
      return std::hash<unsigned long long>()((unsigned long long)v.first * 1000003ull ^
                                             (unsigned long long)v.second);
    }
  };
  std::unordered_set<std::pair<I, I>, hash> seen;
  std::vector<std::pair<std::pair<I, I>, T>> entries;
  std::size_t nnz = density * shape[0] * shape[1];
  entries.reserve(nnz);
  std::mt19937 gen(seed);
  std::uniform_int_distribution<I> row(0, shape[0] - 1);
  std::uniform_int_distribution<I> column(0, shape[1] - 1);
  std::uniform_real_distribution<T> value_gen(0, 1);
  while (seen.size() < nnz) {
    auto i = row(gen);
    auto j = column(gen);
    if (seen.find({i, j}) == seen.end()) {
      T value = value_gen(gen);
      seen.insert({i, j});
      entries.push_back({{i, j}, value});
    }
  }
  T *values = new T[nnz];
  I *rowptr = new I[shape[0] + 1];
  I *colind = new I[nnz];
  std::sort(entries.begin(), entries.end());
  rowptr[0] = 0;
  std::size_t r = 0, c = 0;
  for (auto &[ij, v] : entries) {
    values[c] = v;
    colind[c] = ij.second;
    while (r < (std::size_t)ij.first) {
      rowptr[r + 1] = (I)c;
      r++;
    }
    c++;
  }
  for (; r < (std::size_t)shape[0]; r++)
    rowptr[r + 1] = (I)nnz;
  return views::csr_matrix_view<T, I>(values, rowptr, colind, shape, nnz, 0);
}

template <typename T = float, std::integral I = std::size_t>
auto generate_band_csr(I size, std::size_t up_band = 3,
                       std::size_t down_band = 3) {
  std::size_t nnz = (1 + up_band + down_band) * size -
                    (up_band * (up_band + 1) / 2) -
                    (down_band * (down_band + 1) / 2);
  T *values = new T[nnz];
  I *rowptr = new I[size + 1];
  I *colind = new I[nnz];
  rowptr[0] = 0;
  std::size_t c = 0;
  for (long long i = 0; i < (long long)size; i++) {
    for (long long j = std::max(i - (long long)down_band, 0ll); j < i; j++) {
      values[c] = 1;
      colind[c++] = (I)j;
    }
    values[c] = 1;
    colind[c++] = (I)i;
    for (long long j = i + 1; j <= i + (long long)up_band; j++) {
      if (j >= (long long)size)
        continue;
      values[c] = 1;
      colind[c++] = (I)j;
    }
    rowptr[i + 1] = (I)c;
  }
  return views::csr_matrix_view<T, I>(values, rowptr, colind, {size, size},
                                      nnz, 0);
}

// dr::read_csr<T, I>(path, one_indexed) (include/dr/detail/matrix_io.hpp:
// 246-256): a coordinate Matrix Market file, parsed by the library
// (drb_read_matrix_market), as a host view with arrays owned by the caller
// (free with __detail::destroy_csr_matrix_view).  Errors throw
// std::runtime_error with the reference's messages.
template <typename T, typename I = std::size_t>
auto read_csr(std::string file_path, bool one_indexed = true) {
  drb_csr_host h{};
  if (drb_read_matrix_market(file_path.c_str(), one_indexed ? 1 : 0, &h) !=
      DRB_OK)
    throw std::runtime_error(drb_last_error());
  T *values = new T[h.nnz > 0 ? h.nnz : 1];
  I *rowptr = new I[h.m + 1];
  I *colind = new I[h.nnz > 0 ? h.nnz : 1];
  for (int64_t i = 0; i <= h.m; i++)
    rowptr[i] = (I)h.rowptr[i];
  for (int64_t k = 0; k < h.nnz; k++) {
    colind[k] = (I)h.colind[k];
    values[k] = (T)h.values[k];
  }
  const index<I> shape((I)h.m, (I)h.n);
  const std::size_t nnz = (std::size_t)h.nnz;
  drb_csr_host_free(&h);
  return views::csr_matrix_view<T, I>(values, rowptr, colind, shape, nnz, 0);
}

namespace __detail {
// Frees a view made by the generators or read_csr (matrix_io.hpp:235-243).
template <typename T, typename I, typename A = std::allocator<T>>
void destroy_csr_matrix_view(views::csr_matrix_view<T, I> view, A = A{}) {
  delete[] view.values_data();
  delete[] view.rowptr_data();
  delete[] view.colind_data();
}
} // namespace __detail

namespace mp {

// ---- runtime ---------------------------------------------------------------------
struct communicator {
  int rank() const { return 0; }
  int size() const { return 1; }
};
inline communicator default_comm() { return {}; }
inline void init() {}
inline void finalize() { check(drb_stream_synchronize(nullptr)); }
inline bool use_sycl() { return false; }
struct MpiBackend {}; // backend tag kept for template-argument compatibility

struct distribution {
  std::size_t prev = 0, next = 0, gran = 1;
  bool periodic_ = false;
  distribution &halo(std::size_t radius) {
    prev = next = radius;
    return *this;
  }
  distribution &halo(std::size_t p, std::size_t n) {
    prev = p;
    next = n;
    return *this;
  }
  distribution &periodic(bool p) {
    periodic_ = p;
    return *this;
  }
  distribution &granularity(std::size_t g) {
    gran = g;
    return *this;
  }
  std::size_t granularity() const { return gran; }
};

// Device buffer owned by the C ABI's allocator.
template <class T> class device_buffer {
public:
  device_buffer() = default;
  explicit device_buffer(std::size_t n) { allocate(n); }
  device_buffer(const device_buffer &) = delete;
  device_buffer &operator=(const device_buffer &) = delete;
  device_buffer(device_buffer &&o) noexcept { swap(o); }
  device_buffer &operator=(device_buffer &&o) noexcept {
    swap(o);
    return *this;
  }
  ~device_buffer() { release(); }
  void allocate(std::size_t n) {
    release();
    void *p = nullptr;
    check(drb_malloc(&p, sizeof(T) * std::max<std::size_t>(n, 1)));
    ptr_ = static_cast<T *>(p);
    n_ = n;
  }
  void release() {
    if (ptr_)
      drb_free(ptr_);
    ptr_ = nullptr;
    n_ = 0;
  }
  T *data() const { return ptr_; }
  std::size_t size() const { return n_; }
  void upload(const T *host, std::size_t n, std::size_t offset = 0) {
    check(drb_memcpy(ptr_ + offset, host, sizeof(T) * n, 0, nullptr));
    check(drb_stream_synchronize(nullptr));
  }
  void download(T *host, std::size_t n, std::size_t offset = 0) const {
    check(drb_memcpy(host, ptr_ + offset, sizeof(T) * n, 1, nullptr));
    check(drb_stream_synchronize(nullptr));
  }

private:
  void swap(device_buffer &o) {
    std::swap(ptr_, o.ptr_);
    std::swap(n_, o.n_);
  }
  T *ptr_ = nullptr;
  std::size_t n_ = 0;
};

// Replicated x (broadcasted_vector.hpp:9-51): one device copy.
template <typename T> class broadcasted_vector {
public:
  broadcasted_vector() = default;
  template <std::ranges::input_range R>
  void broadcast_data(std::size_t data_size, std::size_t root, R root_data,
                      communicator = default_comm()) {
    if (root != 0)
      throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
    std::vector<T> tmp(std::ranges::begin(root_data), std::ranges::end(root_data));
    tmp.resize(data_size);
    buf_.allocate(data_size);
    buf_.upload(tmp.data(), data_size);
  }
  void destroy_data() { buf_.release(); }
  T operator[](std::size_t i) const {
    T v;
    buf_.download(&v, 1, i);
    return v;
  }
  T *broadcasted_data() { return buf_.data(); }
  std::size_t size() const { return buf_.size(); }

private:
  device_buffer<T> buf_;
};

// k replicated right-hand sides, column-major (broadcasted_slim_matrix.hpp).
template <typename T> class broadcasted_slim_matrix {
public:
  broadcasted_slim_matrix() = default;
  void broadcast_data(std::size_t height, std::size_t width, std::size_t root,
                      T **root_data, communicator = default_comm()) {
    if (root != 0)
      throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
    height_ = height;
    width_ = width;
    buf_.allocate(height * width);
    for (std::size_t i = 0; i < width; i++)
      buf_.upload(root_data[i], height, height * i);
  }
  template <std::ranges::input_range R>
  void broadcast_data(std::size_t height, std::size_t width, std::size_t root,
                      R root_data, communicator = default_comm()) {
    if (root != 0)
      throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
    std::vector<T> tmp(std::ranges::begin(root_data), std::ranges::end(root_data));
    tmp.resize(height * width);
    height_ = height;
    width_ = width;
    buf_.allocate(height * width);
    buf_.upload(tmp.data(), height * width);
  }
  void destroy_data() { buf_.release(); }
  T *broadcasted_data() { return buf_.data(); }
  std::size_t width() const { return width_; }

private:
  device_buffer<T> buf_;
  std::size_t height_ = 0, width_ = 0;
};

// ---- distributions: own the device-resident matrix through a drb_csr_t -----
template <typename T, typename I, class BackendT, drb_partition Part>
class csr_distribution_base {
public:
  using value_type = matrix_entry<T, I>;
  using elem_type = T;
  using index_type = I;
  using difference_type = std::ptrdiff_t;

  struct segment_info {
    std::size_t rank;
    std::int64_t row_begin, row_end, nnz_begin, nnz_end;
    std::size_t size() const { return (std::size_t)(nnz_end - nnz_begin); }
  };

  csr_distribution_base(const csr_distribution_base &) = delete;
  csr_distribution_base &operator=(const csr_distribution_base &) = delete;

  csr_distribution_base(views::csr_matrix_view<T, I> csr_view,
                        distribution dist = distribution(), std::size_t root = 0,
                        int nsegments = 1, uint32_t flags = 0)
      : dist_(dist) {
    if (root != 0)
      throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
    shape_ = {(std::size_t)csr_view.shape()[0], (std::size_t)csr_view.shape()[1]};
    nnz_ = csr_view.size();
    check(drb_csr_create(&h_, (int64_t)shape_[0], (int64_t)shape_[1],
                         (int64_t)nnz_, csr_view.rowptr_data(),
                         csr_view.colind_data(), csr_view.values_data(),
                         detail::itype_of<I>(), detail::dtype_of<T>(),
                         detail::dtype_of<T>(), nsegments, Part, flags, nullptr));
    int ns = 0;
    check(drb_csr_num_segments(h_, &ns));
    for (int s = 0; s < ns; s++) {
      segment_info si{(std::size_t)s, 0, 0, 0, 0};
      check(drb_csr_segment(h_, s, &si.row_begin, &si.row_end, &si.nnz_begin,
                            &si.nnz_end));
      segs_.push_back(si);
      offsets_.push_back((std::size_t)si.nnz_begin);
    }
  }
  ~csr_distribution_base() {
    if (h_)
      drb_csr_destroy(h_);
  }

  std::size_t nnz() const { return nnz_; }
  index<std::size_t> shape() const { return shape_; }
  void fence() const { check(drb_stream_synchronize(nullptr)); }
  const std::vector<segment_info> &segments() const { return segs_; }
  std::size_t get_segment_from_offset(std::size_t offset) const {
    auto it = std::upper_bound(offsets_.begin(), offsets_.end(), offset);
    return (std::size_t)(it - offsets_.begin()) - 1;
  }
  std::size_t get_id_in_segment(std::size_t offset) const {
    return offset - offsets_[get_segment_from_offset(offset)];
  }
  drb_csr_t handle() const { return h_; }

  value_type entry(std::size_t offset) const {
    int64_t r, c;
    double v;
    check(drb_csr_get_entries(h_, (int64_t)offset, 1, &r, &c, &v));
    return value_type(index<I>((I)r, (I)c), (T)v);
  }

  // local_gemv_and_collect (csr_row_distribution.hpp:137-153): y = A x for
  // `width` column-major right-hand sides; x is device memory (the
  // broadcasted data); res receives m*width values on root.
  template <typename C>
  void local_gemv_and_collect(std::size_t root, C &res, T *x,
                              std::size_t width) const {
    assert(std::ranges::size(res) == shape_.first * width);
    if (root != 0)
      throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
    const std::size_t count = shape_.first * width;
    if (ybuf_.size() < count)
      ybuf_.allocate(count);
    check(drb_csr_gemv(h_, x, ybuf_.data(), (int64_t)width, DRB_COL_MAJOR, nullptr));
    std::vector<T> host(count);
    ybuf_.download(host.data(), count);
    std::ranges::copy(host, std::ranges::begin(res));
  }

private:
  drb_csr_t h_ = nullptr;
  distribution dist_;
  index<std::size_t> shape_;
  std::size_t nnz_ = 0;
  std::vector<segment_info> segs_;
  std::vector<std::size_t> offsets_;
  mutable device_buffer<T> ybuf_;
};

template <typename T, typename I, class BackendT = MpiBackend>
class csr_row_distribution
    : public csr_distribution_base<T, I, BackendT, DRB_PART_ROW> {
  using base = csr_distribution_base<T, I, BackendT, DRB_PART_ROW>;

public:
  using base::base;
};

template <typename T, typename I, class BackendT = MpiBackend>
class csr_eq_distribution
    : public csr_distribution_base<T, I, BackendT, DRB_PART_EQ> {
  using base = csr_distribution_base<T, I, BackendT, DRB_PART_EQ>;

public:
  using base::base;
};

template <typename T>
concept vector_multiplicable =
    requires(T t, std::vector<typename T::elem_type> res,
             typename T::elem_type *input) {
      t.local_gemv_and_collect(int(), res, input, 1);
    };

// distributed_sparse_matrix (distributed_sparse_matrix.hpp:29-162).
template <typename T, typename I, class BackendT = MpiBackend,
          class MatrixDistrT = csr_eq_distribution<T, I, BackendT>>
class distributed_sparse_matrix {
public:
  using value_type = matrix_entry<T, I>;
  using elem_type = T;
  using index_type = I;
  using key_type = index<I>;
  using size_type = std::size_t;
  using difference_type = std::ptrdiff_t;
  using backend_type = BackendT;

  class iterator {
  public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type = typename distributed_sparse_matrix::value_type;
    using difference_type = std::ptrdiff_t;
    iterator() = default;
    iterator(const distributed_sparse_matrix *p, difference_type o)
        : parent_(p), offset_(o) {}
    value_type operator*() const { return parent_->distribution_.entry(offset_); }
    value_type operator[](difference_type n) const { return *(*this + n); }
    iterator operator+(difference_type n) const { return {parent_, offset_ + n}; }
    friend iterator operator+(difference_type n, const iterator &it) { return it + n; }
    iterator operator-(difference_type n) const { return {parent_, offset_ - n}; }
    difference_type operator-(const iterator &o) const { return offset_ - o.offset_; }
    iterator &operator+=(difference_type n) {
      offset_ += n;
      return *this;
    }
    iterator &operator-=(difference_type n) {
      offset_ -= n;
      return *this;
    }
    iterator &operator++() {
      ++offset_;
      return *this;
    }
    iterator operator++(int) {
      auto o = *this;
      ++offset_;
      return o;
    }
    iterator &operator--() {
      --offset_;
      return *this;
    }
    iterator operator--(int) {
      auto o = *this;
      --offset_;
      return o;
    }
    bool operator==(const iterator &o) const {
      return parent_ == o.parent_ && offset_ == o.offset_;
    }
    auto operator<=>(const iterator &o) const { return offset_ <=> o.offset_; }

  private:
    const distributed_sparse_matrix *parent_ = nullptr;
    difference_type offset_ = 0;
  };

  distributed_sparse_matrix(const distributed_sparse_matrix &) = delete;
  distributed_sparse_matrix &operator=(const distributed_sparse_matrix &) = delete;

  distributed_sparse_matrix(views::csr_matrix_view<T, I> csr_view,
                            std::size_t root = 0,
                            distribution dist = distribution(), int nsegments = 1,
                            uint32_t flags = 0)
      : distribution_(csr_view, dist, root, nsegments, flags) {}

  iterator begin() const { return iterator(this, 0); }
  iterator end() const { return begin() + (difference_type)distribution_.nnz(); }
  std::size_t size() const { return distribution_.nnz(); }
  auto shape() const { return distribution_.shape(); }
  value_type operator[](difference_type n) const { return *(begin() + n); }
  const auto &segments() const { return distribution_.segments(); }
  void fence() { distribution_.fence(); }
  drb_csr_t handle() const { return distribution_.handle(); }

  template <typename C>
  void local_gemv_and_collect(std::size_t root, C &res, T *vals,
                              std::size_t val_width) const {
    distribution_.local_gemv_and_collect(root, res, vals, val_width);
  }

private:
  MatrixDistrT distribution_;
};

// ---- gemv (gemv.hpp:16-71) ---------------------------------------------------------
template <typename T, typename I, std::ranges::output_range<T> C, typename Backend,
          typename MatDistr>
  requires(vector_multiplicable<MatDistr>)
void gemv(int root, C &res, distributed_sparse_matrix<T, I, Backend, MatDistr> &a,
          broadcasted_vector<T> &b) {
  if (default_comm().rank() == root) {
    assert(a.shape().first == std::ranges::size(res));
    assert(a.shape().second == b.size());
  }
  a.local_gemv_and_collect(root, res, b.broadcasted_data(), 1);
}

template <typename T, typename I, std::ranges::output_range<T> C, typename Backend,
          typename MatDistr>
  requires(vector_multiplicable<MatDistr>)
void gemv(int root, C &res, distributed_sparse_matrix<T, I, Backend, MatDistr> &a,
          broadcasted_slim_matrix<T> &b) {
  if (default_comm().rank() == root)
    assert(a.shape().first * b.width() == std::ranges::size(res));
  a.local_gemv_and_collect(root, res, b.broadcasted_data(), b.width());
}

template <typename T, typename I, std::ranges::output_range<T> C, typename Backend,
          typename MatDistr>
  requires(vector_multiplicable<MatDistr>)
void gemv(C &res, distributed_sparse_matrix<T, I, Backend, MatDistr> &a,
          broadcasted_vector<T> &b) {
  gemv(0, res, a, b); // one rank: the root's result is everyone's
}

template <typename T, typename I, std::ranges::output_range<T> C, typename Backend,
          typename MatDistr>
  requires(vector_multiplicable<MatDistr>)
void gemv(C &res, distributed_sparse_matrix<T, I, Backend, MatDistr> &a,
          broadcasted_slim_matrix<T> &b) {
  gemv(0, res, a, b);
}

// ---- distributed_vector, iota, fill, reduce ---------------------------------------
namespace detail {
template <class T> constexpr drb_dtype vec_dtype_of() {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double> ||
                    (std::is_integral_v<T> && std::is_signed_v<T> &&
                     (sizeof(T) == 4 || sizeof(T) == 8)),
                "distributed_vector element type: float, double, int32 or int64");
  if constexpr (std::is_same_v<T, float>)
    return DRB_F32;
  else if constexpr (std::is_same_v<T, double>)
    return DRB_F64;
  else
    return sizeof(T) == 4 ? DRB_INT32 : DRB_INT64;
}
} // namespace detail

// distributed_vector<T> (distributed_vector.hpp:150-340) on one GPU: all n
// elements in one device buffer; segment r covers [r*ceil(n/P), ...) as
// segment_size does (distributed_vector.hpp:310), P = nsegments.  Elements
// are read and written through get()/put() (host copies).
template <typename T, class BackendT = MpiBackend> class distributed_vector {
public:
  using value_type = T;
  using size_type = std::size_t;
  using difference_type = std::ptrdiff_t;
  using backend_type = BackendT;

  struct segment {
    std::size_t rank_, begin_, end_;
    std::size_t rank() const { return rank_; }
    std::size_t size() const { return end_ - begin_; }
    std::size_t begin() const { return begin_; }
    std::size_t end() const { return end_; }
  };

  class iterator {
  public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type = T;
    using difference_type = std::ptrdiff_t;
    iterator() = default;
    iterator(const distributed_vector *p, difference_type o) : parent_(p), offset_(o) {}
    T operator*() const { return parent_->get((std::size_t)offset_); }
    T operator[](difference_type n) const { return *(*this + n); }
    iterator operator+(difference_type n) const { return {parent_, offset_ + n}; }
    friend iterator operator+(difference_type n, const iterator &it) { return it + n; }
    iterator operator-(difference_type n) const { return {parent_, offset_ - n}; }
    difference_type operator-(const iterator &o) const { return offset_ - o.offset_; }
    iterator &operator+=(difference_type n) {
      offset_ += n;
      return *this;
    }
    iterator &operator-=(difference_type n) {
      offset_ -= n;
      return *this;
    }
    iterator &operator++() {
      ++offset_;
      return *this;
    }
    iterator operator++(int) {
      auto o = *this;
      ++offset_;
      return o;
    }
    iterator &operator--() {
      --offset_;
      return *this;
    }
    iterator operator--(int) {
      auto o = *this;
      --offset_;
      return o;
    }
    bool operator==(const iterator &o) const {
      return parent_ == o.parent_ && offset_ == o.offset_;
    }
    auto operator<=>(const iterator &o) const { return offset_ <=> o.offset_; }
    const distributed_vector *parent() const { return parent_; }
    difference_type offset() const { return offset_; }

  private:
    const distributed_vector *parent_ = nullptr;
    difference_type offset_ = 0;
  };

  distributed_vector(const distributed_vector &) = delete;
  distributed_vector &operator=(const distributed_vector &) = delete;
  explicit distributed_vector(std::size_t size = 0, distribution = distribution(),
                              int nsegments = 1)
      : n_(size), nseg_(std::max(1, nsegments)) {
    buf_.allocate(size);
  }
  distributed_vector(std::size_t size, value_type fill_value,
                     distribution = distribution(), int nsegments = 1)
      : distributed_vector(size, distribution(), nsegments) {
    check(drb_fill((int64_t)n_, buf_.data(), detail::vec_dtype_of<T>(), &fill_value,
                   nullptr));
  }

  std::size_t size() const { return n_; }
  iterator begin() const { return iterator(this, 0); }
  iterator end() const { return iterator(this, (difference_type)n_); }
  T *data() const { return buf_.data(); }
  std::size_t segment_size() const { return (n_ + nseg_ - 1) / (std::size_t)nseg_; }
  std::vector<segment> segments() const {
    std::vector<segment> out;
    const std::size_t seg = segment_size();
    for (std::size_t r = 0; r < (std::size_t)nseg_; r++)
      out.push_back({r, std::min(n_, r * seg), std::min(n_, (r + 1) * seg)});
    return out;
  }
  T get(std::size_t i) const {
    T v;
    buf_.download(&v, 1, i);
    return v;
  }
  void put(std::size_t i, T v) { buf_.upload(&v, 1, i); }
  T operator[](std::size_t i) const { return get(i); }
  void fence() { check(drb_stream_synchronize(nullptr)); }

private:
  std::size_t n_;
  int nseg_;
  device_buffer<T> buf_;
};

// Reduction operators the device reduce runs: std::plus, and min / max (the
// reference tests pass min/max lambdas; name them here instead).
namespace ops {
struct min {
  template <class A, class B> auto operator()(A a, B b) const { return b < a ? b : a; }
};
struct max {
  template <class A, class B> auto operator()(A a, B b) const { return a < b ? b : a; }
};
} // namespace ops

namespace detail {
template <class O> struct is_plus : std::false_type {};
template <class T> struct is_plus<std::plus<T>> : std::true_type {};
template <class Op> constexpr drb_reduce_op reduce_op_of() {
  using O = std::remove_cvref_t<Op>;
  if constexpr (std::is_same_v<O, ops::min>)
    return DRB_REDUCE_MIN;
  else if constexpr (std::is_same_v<O, ops::max>)
    return DRB_REDUCE_MAX;
  else {
    static_assert(is_plus<O>::value, "drb::mp::reduce runs std::plus, drb::mp::ops::min "
                                     "or drb::mp::ops::max on the GPU");
    return DRB_REDUCE_SUM;
  }
}

// One reduce over [first, last) of v; the device result is copied back.
template <class V, class Op>
typename V::value_type reduce_span(const V &v, std::size_t first, std::size_t last,
                                   const typename V::value_type *init, Op &&) {
  using E = typename V::value_type;
  device_buffer<E> out(1);
  check(drb_reduce((int64_t)(last - first), v.data() + first, vec_dtype_of<E>(),
                   reduce_op_of<Op>(), init, out.data(), nullptr));
  E r;
  out.download(&r, 1);
  return r;
}
} // namespace detail

// reduce over ranges (reduce.hpp:127-181) ...
template <typename T, typename E, class B, typename Op>
T reduce(std::size_t root, const distributed_vector<E, B> &r, T init, Op &&op) {
  if (root != 0)
    throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
  const E i = static_cast<E>(init);
  return static_cast<T>(detail::reduce_span(r, 0, r.size(), &i, op));
}
template <typename T, typename E, class B, typename Op>
T reduce(const distributed_vector<E, B> &r, T init, Op &&op) {
  return ::drb::mp::reduce(0, r, init, op);
}
template <typename T, typename E, class B>
T reduce(std::size_t root, const distributed_vector<E, B> &r, T init) {
  return ::drb::mp::reduce(root, r, init, std::plus<>{});
}
template <typename T, typename E, class B>
T reduce(const distributed_vector<E, B> &r, T init) {
  return ::drb::mp::reduce(0, r, init, std::plus<>{});
}
template <typename E, class B>
E reduce(std::size_t root, const distributed_vector<E, B> &r) {
  if (root != 0)
    throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
  return detail::reduce_span(r, 0, r.size(), nullptr, std::plus<>{});
}
template <typename E, class B> E reduce(const distributed_vector<E, B> &r) {
  return ::drb::mp::reduce(0, r);
}

// ... and over iterator pairs (reduce.hpp:183-232).
template <typename It, typename T, typename Op>
  requires requires(It it) { it.parent()->data(); }
auto reduce(std::size_t root, It first, It last, T init, Op &&op) {
  if (root != 0)
    throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
  using V = std::remove_cvref_t<decltype(*first.parent())>;
  using E = typename V::value_type;
  const E i = static_cast<E>(init);
  return static_cast<T>(detail::reduce_span(*first.parent(), (std::size_t)first.offset(),
                                            (std::size_t)last.offset(), &i, op));
}
template <typename It, typename T>
  requires requires(It it) { it.parent()->data(); }
auto reduce(std::size_t root, It first, It last, T init) {
  return ::drb::mp::reduce(root, first, last, init, std::plus<>{});
}
template <typename It>
  requires requires(It it) { it.parent()->data(); }
auto reduce(std::size_t root, It first, It last) {
  if (root != 0)
    throw error(DRB_ERR_INVALID_ARG, "drb: root is not a rank");
  return detail::reduce_span(*first.parent(), (std::size_t)first.offset(),
                             (std::size_t)last.offset(), nullptr, std::plus<>{});
}
template <typename It, typename T, typename Op>
  requires requires(It it) { it.parent()->data(); }
auto reduce(It first, It last, T init, Op &&op) {
  using V = std::remove_cvref_t<decltype(*first.parent())>;
  using E = typename V::value_type;
  const E i = static_cast<E>(init);
  return static_cast<T>(detail::reduce_span(*first.parent(), (std::size_t)first.offset(),
                                            (std::size_t)last.offset(), &i, op));
}
template <typename It, typename T>
  requires requires(It it) { it.parent()->data(); }
auto reduce(It first, It last, T init) {
  return ::drb::mp::reduce(first, last, init, std::plus<>{});
}
template <typename It>
  requires requires(It it) { it.parent()->data(); }
auto reduce(It first, It last) {
  return detail::reduce_span(*first.parent(), (std::size_t)first.offset(),
                             (std::size_t)last.offset(), nullptr, std::plus<>{});
}

// iota / fill (iota.hpp:20-34, fill.hpp:21-30)
template <typename E, class B, std::integral T>
void iota(distributed_vector<E, B> &r, T value) {
  check(drb_iota((int64_t)r.size(), r.data(), detail::vec_dtype_of<E>(), (int64_t)value,
                 nullptr));
}
template <typename It, std::integral T>
  requires requires(It it) { it.parent()->data(); }
void iota(It first, It last, T value) {
  using V = std::remove_cvref_t<decltype(*first.parent())>;
  check(drb_iota((int64_t)(last - first), first.parent()->data() + first.offset(),
                 detail::vec_dtype_of<typename V::value_type>(), (int64_t)value, nullptr));
}
template <typename E, class B, typename T>
auto fill(distributed_vector<E, B> &r, T value) {
  const E v = static_cast<E>(value);
  check(drb_fill((int64_t)r.size(), r.data(), detail::vec_dtype_of<E>(), &v, nullptr));
  return r.end();
}
template <typename It, typename T>
  requires requires(It it) { it.parent()->data(); }
auto fill(It first, It last, T value) {
  using V = std::remove_cvref_t<decltype(*first.parent())>;
  using E = typename V::value_type;
  const E v = static_cast<E>(value);
  check(drb_fill((int64_t)(last - first), first.parent()->data() + first.offset(),
                 detail::vec_dtype_of<E>(), &v, nullptr));
  return last;
}

// ---- conjugate gradients on the device (drb_csr_cg) ------------------------------
// Solves a x = b for symmetric positive definite a; x holds the initial guess.
template <typename T, typename I, class B, class D>
drb_cg_info conjugate_gradient(distributed_sparse_matrix<T, I, B, D> &a,
                               const distributed_vector<T, B> &b, distributed_vector<T, B> &x,
                               int64_t max_iters = 1000, double rtol = 1e-8) {
  drb_cg_info info{};
  check(drb_csr_cg(a.handle(), b.data(), x.data(), max_iters, rtol, &info, nullptr));
  return info;
}

} // namespace mp
} // namespace drb

// Structured bindings: auto [i, j] = idx; auto [index, value] = entry;
template <std::integral T>
struct std::tuple_size<drb::index<T>> : std::integral_constant<std::size_t, 2> {};
template <std::size_t N, std::integral T> struct std::tuple_element<N, drb::index<T>> {
  using type = T;
};
template <typename T, std::integral I>
struct std::tuple_size<drb::matrix_entry<T, I>> : std::integral_constant<std::size_t, 2> {};
template <typename T, std::integral I> struct std::tuple_element<0, drb::matrix_entry<T, I>> {
  using type = drb::index<I>;
};
template <typename T, std::integral I> struct std::tuple_element<1, drb::matrix_entry<T, I>> {
  using type = T;
};
