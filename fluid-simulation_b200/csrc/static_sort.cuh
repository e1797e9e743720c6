// static_sort.cuh — the allocation-free key sort behind wcsph_sort_keys_static.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace wcsph {

// Enqueues on `stream` the stable sort permutation of n <= WCSPH_STATIC_SORT_MAX_KEYS
// device-resident keys into the device array perm (throws Error on bad input).
void static_sort_permutation(const uint64_t* keys, uint32_t n, uint32_t* perm, cudaStream_t stream);

}  // namespace wcsph
