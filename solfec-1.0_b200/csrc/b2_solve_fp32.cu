// b2_solve_fp32.cu -- the FP32 sweeps of mixed precision in their own
// translation unit, built with fused multiply-adds (the rest of the library
// is built without them, so that its FP64 arithmetic rounds exactly as the
// reference's C code does). The kernel body is that of k_solve<true>
// (b2_solve.cuh); only the contraction of multiplies and adds differs.
#include <cuda_runtime.h>
#include "b2_solve.cuh"

namespace b2 {

__global__ void __launch_bounds__(kSolveThreads, 6) k_solve_fp32(const __grid_constant__ SolveArgs a) {
  solve_persistent<true, false>(a);
}

__global__ void __launch_bounds__(kSolveThreads, 6) k_solve_fp32_kinds(const __grid_constant__ SolveArgs a) {
  solve_persistent<true, true>(a);
}

}  // namespace b2
