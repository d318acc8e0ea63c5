// k_lines_fast.cu -- tiled line solver, fast build: FMA contraction and
// multiplication by tabulated reciprocals on mask-free lines (results agree
// with the reference-exact build to a few ulps per sweep).
#include "k_lines.cuh"

namespace nse {

template <int DIR, int KIND>
static void go(const Dims& d, double* f, const LineArgs& a, const LineTab& tb, const int* slots,
               const double* ltab, cudaStream_t s) {
  int n = DIR == 0 ? d.nx : (DIR == 1 ? d.ny : d.nz);
  int pitch = (n + 2) | 1;
  size_t sm = 32 * (size_t)pitch * sizeof(double);
  auto kern = k_lines<DIR, KIND, false>;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int nl = DIR == 0 ? a.jtop : d.nx;
  int other = DIR == 1 ? d.nz : (DIR == 2 ? a.jtop : d.nz);
  dim3 grid((nl + 31) / 32, other);
  count_launch();
  kern<<<grid, 32, sm, s>>>(d, f, a, tb, slots, ltab, pitch);
}

void launch_lines_fast(int dir, int kind, const Dims& d, double* f, const LineArgs& a,
                       const LineTab& tb, const int* slots, const double* ltab,
                       cudaStream_t s) {
  if (dir == 1) {
    if (kind == LK_UL_U) go<1, LK_UL_U>(d, f, a, tb, slots, ltab, s);
    else if (kind == LK_UL_V) go<1, LK_UL_V>(d, f, a, tb, slots, ltab, s);
    else go<1, LK_UL_T>(d, f, a, tb, slots, ltab, s);
  } else if (dir == 2) {
    if (kind == LK_CYC_VEL) go<2, LK_CYC_VEL>(d, f, a, tb, slots, ltab, s);
    else go<2, LK_CYC_T>(d, f, a, tb, slots, ltab, s);
  } else {
    if (kind == LK_CYC_VEL) go<0, LK_CYC_VEL>(d, f, a, tb, slots, ltab, s);
    else go<0, LK_CYC_T>(d, f, a, tb, slots, ltab, s);
  }
}

}  // namespace nse
