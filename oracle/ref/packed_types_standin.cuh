/* Stand-in for hpc_helpers' packed_types.cuh: the reference headers only
 * name these two templates, with integer bit-width arguments, inside
 * out-of-scope multi-value storage types that the golden programs never
 * instantiate. */
#ifndef WC_REF_PACKED_TYPES_STANDIN
#define WC_REF_PACKED_TYPES_STANDIN
#include <cstdint>
namespace packed_types {
template <std::uint64_t A, std::uint64_t B> class PackedPair;
template <std::uint64_t A, std::uint64_t B, std::uint64_t C, std::uint64_t D>
class PackedQuadruple;
}
#endif
