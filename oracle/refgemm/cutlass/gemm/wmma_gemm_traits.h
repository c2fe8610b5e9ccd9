// Test infrastructure (oracle side): the traits and epilogue names of
// CUTLASS 1.3 that src/helper.cu:716-730 of hiperbio/tensor-episdet
// instantiates.  Only the parameters that define the arithmetic are kept
// (operand layouts and types, the output type, the linear-scaling epilogue);
// the tile shapes only tuned the original kernel and are accepted and ignored.
#pragma once
#include "../wmma_matrix.h"

namespace cutlass {
namespace gemm {

// D = alpha * (A x B) + beta * C.
template <typename Scalar_>
struct LinearScaling {
    typedef Scalar_ Scalar;
};

template <MatrixLayout::Kind kLayoutA_, MatrixLayout::Kind kLayoutB_, typename OutputTile_, typename ScalarA_,
          typename ScalarB_, typename ScalarD_, typename Epilogue_, typename Accumulator_, typename WarpTile_,
          typename InstructionShape_, int kScalarsPerLdgA_, int kScalarsPerLdgB_>
struct WmmaGemmTraits {
    static constexpr MatrixLayout::Kind kLayoutA = kLayoutA_;
    static constexpr MatrixLayout::Kind kLayoutB = kLayoutB_;
    typedef ScalarA_ ScalarA;
    typedef ScalarB_ ScalarB;
    typedef ScalarD_ ScalarD;
    typedef ScalarD_ ScalarC;
    typedef Epilogue_ Epilogue;
};

}  // namespace gemm
}  // namespace cutlass
