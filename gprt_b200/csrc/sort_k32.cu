// sort_k32.cu -- every shape of the sort's tuning grid for uint32_t keys (no payload).
#include "sort_kernels.cuh"

namespace gprtcu {
const std::array<SortRunFn, kSortGridSize> kSortTableK32 =
    make_sort_table<uint32_t, char>(std::make_index_sequence<kSortGridSize>{});
}  // namespace gprtcu
