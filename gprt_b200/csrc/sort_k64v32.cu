// sort_k64v32.cu -- every shape of the sort's tuning grid for uint64_t keys with uint32_t payloads.
#include "sort_kernels.cuh"

namespace gprtcu {
const std::array<SortRunFn, kSortGridSize> kSortTableK64V32 =
    make_sort_table<uint64_t, uint32_t>(std::make_index_sequence<kSortGridSize>{});
}  // namespace gprtcu
