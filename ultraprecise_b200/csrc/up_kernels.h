// up_kernels.h — launchers of the precompiled (nvcc, sm_100a) kernels.
#ifndef UP_KERNELS_H_
#define UP_KERNELS_H_

#include <cuda_runtime.h>
#include <stdint.h>

namespace upi {

cudaError_t launch_fill_segment_gids(const int32_t* starts, int32_t n_groups, int64_t rows, int32_t* gid,
                                     cudaStream_t s);
cudaError_t launch_division_int64(const uint8_t* sums, const int64_t* counts, int32_t n, uint8_t* out,
                                  cudaStream_t s);
// Synchronises the stream to read the group count back.
cudaError_t launch_group_ids_small_keys(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                        int64_t rows, int32_t* gid, int32_t* n_groups, void* group_keys,
                                        cudaStream_t s);
// The key table only (no per-row ids; UP_KEY_TABLE_ENTRIES entries, the
// group count at entry 131072); the _async form does not synchronise.
cudaError_t launch_group_table_small_keys_async(const void* const* key_cols, const int32_t* key_bytes,
                                                int32_t n_keys, int64_t rows, int32_t* table, void* group_keys,
                                                cudaStream_t s);
cudaError_t launch_group_table_small_keys(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                          int64_t rows, int32_t* table, int32_t* n_groups, void* group_keys,
                                          cudaStream_t s);

}  // namespace upi

#endif
