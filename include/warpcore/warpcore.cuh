/* warpcore/warpcore.cuh -- umbrella header of the C++ drop-in
 * (the reference's include/warpcore/warpcore.cuh) */
#ifndef WARPCORE_B200_CXX_WARPCORE_CUH
#define WARPCORE_B200_CXX_WARPCORE_CUH

#include "single_value_hash_table.cuh"
#include "hash_set.cuh"
#include "counting_hash_table.cuh"
#include "bloom_filter.cuh"
#include "multi_value_hash_table.cuh"
#include "multi_bucket_hash_table.cuh"
#include "bucket_list_hash_table.cuh"

#endif
