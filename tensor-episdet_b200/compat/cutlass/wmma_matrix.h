// Interface stand-in for the two CUTLASS 1.3 names that the reference's
// include/helper.hpp:5-7 and :66 need to compile (cutlass::bin1_t and
// cutlass::Vector), so that the reference's own main (src/tensor-episdet.cu)
// can be compiled unmodified and linked against libepisdet_compat_*.a.  No
// CUTLASS code is here or needed: the reference GEMM that used these types is
// replaced by the library.
#pragma once
#include <cstdint>

namespace cutlass {
struct bin1_t {};
template <typename T, int N>
struct Vector {
    uint32_t storage[(N + 31) / 32];
};
}  // namespace cutlass
