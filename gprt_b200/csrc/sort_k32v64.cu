// sort_k32v64.cu -- every shape of the sort's tuning grid for uint32_t keys with uint64_t payloads.
#include "sort_kernels.cuh"

namespace gprtcu {
const std::array<SortRunFn, kSortGridSize> kSortTableK32V64 =
    make_sort_table<uint32_t, uint64_t>(std::make_index_sequence<kSortGridSize>{});
}  // namespace gprtcu
