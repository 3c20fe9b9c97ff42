// Ranking keys by their bytes on the device (discriminate.rs:103-156, 212-292).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace ef {

// Ranks n keys of `words` 64-bit words each (word-major: keys[w·ld + i], word
// 0 most significant), ordered as unsigned integers: rank[i] the number of
// distinct keys below key i, first[r] the smallest i with rank r. Returns the
// number of distinct keys. If `sorted_rows` is given, it receives the rows in
// key order (stable). All pointers are device memory.
int64_t rank_keys(Context& ctx, const uint64_t* keys, int words, int64_t n, int64_t ld, uint32_t* rank,
                  uint32_t* first, cudaStream_t s, uint32_t* sorted_rows = nullptr);

void thrust_iota(Context& ctx, uint32_t* out, int64_t n, cudaStream_t s);

}  // namespace ef
