// drb/dr_mp.hpp -- drop-in spelling: makes the names a dr::mp gemv user writes
// (dr::mp::distributed_sparse_matrix, dr::mp::csr_row_distribution,
// dr::mp::broadcasted_vector, dr::mp::gemv, dr::generate_random_csr,
// dr::read_csr, dr::views::csr_matrix_view, ...) resolve to this library's B200
// implementation.  Include it instead of <dr/mp.hpp> for the gemv path.
#pragma once
#include "mp.hpp"

namespace dr {
using ::drb::generate_band_csr;
using ::drb::generate_random_csr;
using ::drb::index;
using ::drb::matrix_entry;
using ::drb::read_csr;
namespace views {
using ::drb::views::csr_matrix_view;
}
namespace __detail {
using ::drb::__detail::destroy_csr_matrix_view;
}
namespace mp = ::drb::mp;
} // namespace dr
