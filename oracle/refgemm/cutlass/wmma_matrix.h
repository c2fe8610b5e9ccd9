// Test infrastructure (oracle side): a stand-in for the parts of CUTLASS 1.3
// that hiperbio/tensor-episdet's src/helper.cu compiles against, so that the
// reference's own counting and objective kernels (src/helper.cu:13-698) and
// host drivers (src/search-{pairs,triplets}.cu) can be built and run here as a
// second oracle.  CUTLASS 1.3 is an un-vendored third-party dependency of the
// reference (its Makefile passes -Icutlass; include/helper.hpp:5-7 includes
// these three headers); the only CUTLASS code the reference uses is the 1-bit
// XOR+POPC GEMM behind Cutlass_U1_WmmagemmTN (src/helper.cu:714-750), whose
// published contract gemm/gemm.h restates.  This header holds the type names.
#pragma once
#include <cstdint>

namespace cutlass {

// A 1-bit element; Vector<bin1_t, 32> is one 32-bit word of 32 such elements.
struct bin1_t {};

template <typename T, int N>
struct Vector {
    uint32_t storage[(N + 31) / 32];
};

struct MatrixLayout {
    enum Kind { kRowMajor, kColumnMajor };
};

template <int kD_, int kH_, int kW_, int kC_ = 1>
struct Shape {
    static constexpr int kD = kD_, kH = kH_, kW = kW_, kC = kC_;
};

}  // namespace cutlass
