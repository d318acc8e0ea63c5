// k_lines_exact.cu -- tiled line solver, reference-exact build (no FMA
// contraction), plus the per-row tables of mask-free lines and the per-line
// mask flags.  The tables are built here so their arithmetic matches the
// per-line recurrence of the reference operation for operation.
#include "k_lines.cuh"

namespace nse {

// tables: one thread per (direction, kind) table
__global__ void k_line_tables(int n, const double* D, const double* D12, LineArgs a, int kind,
                              double* base) {
  if (threadIdx.x || blockIdx.x) return;
  const int L = n + 2;
  double *l = base, *dm = base + L, *rdm = base + 2 * L, *up = base + 3 * L, *aa = base + 4 * L,
         *gam = base + 5 * L, *bet = base + 6 * L, *rbet = base + 7 * L, *z = base + 8 * L,
         *den = base + 9 * L;
  switch (kind) {
    case LK_UL_U: build_table<LK_UL_U>(n, D, D12, a, l, dm, rdm, up, aa, gam, bet, rbet, z, den); break;
    case LK_UL_V: build_table<LK_UL_V>(n, D, D12, a, l, dm, rdm, up, aa, gam, bet, rbet, z, den); break;
    case LK_UL_T: build_table<LK_UL_T>(n, D, D12, a, l, dm, rdm, up, aa, gam, bet, rbet, z, den); break;
    case LK_CYC_VEL: build_table<LK_CYC_VEL>(n, D, D12, a, l, dm, rdm, up, aa, gam, bet, rbet, z, den); break;
    default: build_table<LK_CYC_T>(n, D, D12, a, l, dm, rdm, up, aa, gam, bet, rbet, z, den); break;
  }
}

void launch_line_table(int n, const double* D, const double* D12, const LineArgs& a, int kind,
                       double* base, cudaStream_t s) {
  count_launch();
  k_line_tables<<<1, 32, 0, s>>>(n, D, D12, a, kind, base);
}

// flag[line] = 1 if the mask of component comp is non-zero anywhere on it
__global__ void k_line_flags(Dims d, const double* c1, int dir, int comp, int jtop,
                             unsigned char* flags) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int n, i = 0, j = 0, k = 0;
  if (dir == 1) {
    if (t >= (long)d.nx * d.nz) return;
    i = 1 + (int)(t % d.nx); k = 1 + (int)(t / d.nx); n = d.ny;
  } else if (dir == 2) {
    if (t >= (long)d.nx * jtop) return;
    i = 1 + (int)(t % d.nx); j = 1 + (int)(t / d.nx); n = d.nz;
  } else {
    if (t >= (long)jtop * d.nz) return;
    j = 1 + (int)(t % jtop); k = 1 + (int)(t / jtop); n = d.nx;
  }
  unsigned char any = 0;
  for (int r = 1; r <= n; ++r) {
    int ii = dir == 0 ? r : i, jj = dir == 1 ? r : j, kk = dir == 2 ? r : k;
    if (mask_at(d, c1, comp, ii, jj, kk) != 0.0) { any = 1; break; }
  }
  flags[t] = any;
}

void launch_line_flags(const Dims& d, const double* c1, int dir, int comp, int jtop,
                       unsigned char* flags, cudaStream_t s) {
  long n = dir == 1 ? (long)d.nx * d.nz : (dir == 2 ? (long)d.nx * jtop : (long)jtop * d.nz);
  count_launch();
  k_line_flags<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d, c1, dir, comp, jtop, flags);
}

// per-line tables of the lines listed in `ids` (lines that touch the mask):
// one thread per line, same sweep as the mask-free table with the rows of
// this line
template <int DIR, int KIND>
__global__ void k_line_tables_masked(Dims d, GridDev g, const double* c1, LineArgs a,
                                     const int* ids, int count, double* out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  long id = ids[t];
  int i = 0, j = 0, k = 0, n;
  if (DIR == 1) { i = 1 + (int)(id % d.nx); k = 1 + (int)(id / d.nx); n = d.ny; }
  else if (DIR == 2) { i = 1 + (int)(id % d.nx); j = 1 + (int)(id / d.nx); n = d.nz; }
  else { j = 1 + (int)(id % a.jtop); k = 1 + (int)(id / a.jtop); n = d.nx; }
  const int L = n + 2;
  double* b = out + (size_t)t * line_table_stride(KIND, n);
  auto row = [&](int r) { return line_row<DIR, KIND>(d, g, c1, a, i, j, k, r); };
  if (KIND <= LK_UL_T)
    sweep_table<KIND>(n, a, row, b, b + L, b + 2 * L, b + 3 * L, nullptr, nullptr, nullptr,
                      nullptr, nullptr, nullptr);
  else
    sweep_table<KIND>(n, a, row, nullptr, nullptr, nullptr, nullptr, b, b + L, b + 2 * L,
                      b + 3 * L, b + 4 * L, b + 5 * L);
}

void launch_line_tables_masked(int dir, int kind, const Dims& d, const GridDev& g,
                               const double* c1, const LineArgs& a, const int* ids, int count,
                               double* out, cudaStream_t s) {
  if (count <= 0) return;
  unsigned nb = (unsigned)((count + 63) / 64);
  count_launch();
  if (dir == 1) {
    if (kind == LK_UL_U) k_line_tables_masked<1, LK_UL_U><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
    else if (kind == LK_UL_V) k_line_tables_masked<1, LK_UL_V><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
    else k_line_tables_masked<1, LK_UL_T><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
  } else if (dir == 2) {
    if (kind == LK_CYC_VEL) k_line_tables_masked<2, LK_CYC_VEL><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
    else k_line_tables_masked<2, LK_CYC_T><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
  } else {
    if (kind == LK_CYC_VEL) k_line_tables_masked<0, LK_CYC_VEL><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
    else k_line_tables_masked<0, LK_CYC_T><<<nb, 64, 0, s>>>(d, g, c1, a, ids, count, out);
  }
}

template <int DIR, int KIND>
static void go(const Dims& d, double* f, const LineArgs& a, const LineTab& tb, const int* slots,
               const double* ltab, cudaStream_t s) {
  int n = DIR == 0 ? d.nx : (DIR == 1 ? d.ny : d.nz);
  int pitch = (n + 2) | 1;
  size_t sm = 32 * (size_t)pitch * sizeof(double);
  auto kern = k_lines<DIR, KIND, true>;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int nl = DIR == 0 ? a.jtop : d.nx;
  int other = DIR == 1 ? d.nz : (DIR == 2 ? a.jtop : d.nz);
  dim3 grid((nl + 31) / 32, other);
  count_launch();
  kern<<<grid, 32, sm, s>>>(d, f, a, tb, slots, ltab, pitch);
}

void launch_lines_exact(int dir, int kind, const Dims& d, double* f, const LineArgs& a,
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
