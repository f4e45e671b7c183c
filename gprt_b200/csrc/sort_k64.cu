// sort_k64.cu -- every shape of the sort's tuning grid for uint64_t keys (no payload).
#include "sort_kernels.cuh"

namespace gprtcu {
const std::array<SortRunFn, kSortGridSize> kSortTableK64 =
    make_sort_table<uint64_t, char>(std::make_index_sequence<kSortGridSize>{});
}  // namespace gprtcu
