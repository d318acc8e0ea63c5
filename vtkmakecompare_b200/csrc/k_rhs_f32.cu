// k_rhs_f32.cu -- the FP32-storage right-hand-side kernels of the mixed-
// precision form (templates in k_rhs_fast.cuh).  Compiled without FMA
// contraction: with FP32 arithmetic the compiler fused products and sums
// differently in different launch shapes (one shape rounded differently
// from the others by FP32 rounding), and the autotuner needs every shape to
// give the same bits.  The FP64-arithmetic variant (math64) rounds every
// operation separately here too.
#include "k_rhs_fast.cuh"

namespace nse {

int ring_wait_error_f32() { return take_ring_wait_err(); }

// FP32 storage; arithmetic in FP32, or FP64 with math64
void launch_rhs_f32(const Dims& d, const GridDev& g, const GridRcp& rg, const StepParams& sp,
                    const double* u, const double* v, const double* w, const double* T,
                    const float* u_ta, const float* v_ta, const float* w_ta, float* u_pre,
                    float* v_pre, float* w_pre, float* T_pre, const double* c1, float* u_a,
                    float* v_a, float* w_a, float* u_T, bool math64, cudaStream_t s,
                    int shape) {
  if (math64)
    rhs_fast<float, double>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre, v_pre, w_pre,
                            T_pre, c1, u_a, v_a, w_a, u_T, s, shape);
  else
    rhs_fast<float, float>(d, g, rg, sp, u, v, w, T, u_ta, v_ta, w_ta, u_pre, v_pre, w_pre,
                           T_pre, c1, u_a, v_a, w_a, u_T, s, shape);
}

}  // namespace nse
