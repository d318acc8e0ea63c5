// fft_core.cuh -- complex arithmetic, small DFT kernels and the
// register-resident 256-point FFT shared by the transform kernels
// (k_fft.cu: one direction per launch; k_poisson2d.cu: both directions of a
// plane in one cluster launch).
#pragma once

#include <cuda_runtime.h>

namespace nse {

// complex arithmetic on double2 / float2 (CT); CReal<CT>::T is the real type
template <class CT> struct CReal;
template <> struct CReal<double2> { using T = double; };
template <> struct CReal<float2> { using T = float; };
template <class CT>
__device__ __forceinline__ CT mkc(typename CReal<CT>::T x, typename CReal<CT>::T y) {
  CT r;
  r.x = x;
  r.y = y;
  return r;
}
template <class CT>
__device__ __forceinline__ CT cmul(CT a, CT b) {
  return mkc<CT>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class CT>
__device__ __forceinline__ CT cadd(CT a, CT b) { return mkc<CT>(a.x + b.x, a.y + b.y); }
template <class CT>
__device__ __forceinline__ CT csub(CT a, CT b) { return mkc<CT>(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
template <class CT>
__device__ __forceinline__ CT mul_mi(CT a, bool inv) {
  return inv ? mkc<CT>(-a.y, a.x) : mkc<CT>(a.y, -a.x);
}

template <int R, class CT>
struct DftSmall;

template <class CT>
struct DftSmall<2, CT> {
  __device__ static void run(CT* v, bool) {
    CT a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <class CT>
struct DftSmall<4, CT> {
  __device__ static void run(CT* v, bool inv) {
    CT t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    CT t2 = cadd(v[1], v[3]), t3 = mul_mi(csub(v[1], v[3]), inv);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};
template <class CT>
struct DftSmall<3, CT> {
  __device__ static void run(CT* v, bool inv) {
    using RT = typename CReal<CT>::T;
    const RT s = (RT)0.86602540378443864676;  // sin(2 pi/3)
    CT t = cadd(v[1], v[2]);
    CT d = csub(v[1], v[2]);
    CT m = mkc<CT>(v[0].x - RT(0.5) * t.x, v[0].y - RT(0.5) * t.y);
    CT r = mul_mi(mkc<CT>(s * d.x, s * d.y), inv);  // -i s (v1 - v2)
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  }
};
template <class CT>
struct DftSmall<5, CT> {
  __device__ static void run(CT* v, bool inv) {
    using RT = typename CReal<CT>::T;
    const RT c1 = (RT)0.30901699437494742410, c2 = (RT)-0.80901699437494742410;
    const RT s1 = (RT)0.95105651629515357212, s2 = (RT)0.58778525229247312917;
    CT a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
    CT b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
    CT x0 = v[0];
    CT p1 = mkc<CT>(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    CT p2 = mkc<CT>(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    CT q1 = mul_mi(mkc<CT>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), inv);
    CT q2 = mul_mi(mkc<CT>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), inv);
    v[0] = mkc<CT>(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
  }
};

// ------------------------------------------- register FFT of length 256 --
// N = 256 = 16 x 16: with n = 16a + b and k = c + 16e,
//   X[c + 16e] = sum_b W256^(bc) W16^(be) [ sum_a x[16a + b] W16^(ac) ].
// Sixteen threads run one transform: thread b holds x[16a + b] (a = 0..15),
// does the inner 16-point DFT in registers, multiplies by W256^(bc), and the
// values are exchanged through shared memory so that thread c holds the 16
// partial sums of its c; the outer 16-point DFT leaves X[c + 16e] in its
// register e.  One exchange and no block-wide barrier per transform (the
// x kernels synchronise a warp, the z kernel its CTA).
// W16^m = exp(-2 pi i m/16) for the products m = a1*e0 of the 4 x 4 split
template <class CT>
__device__ __forceinline__ CT w16(int m, bool inv) {
  using RT = typename CReal<CT>::T;
  const RT c1 = (RT)0.92387953251128675613, s1 = (RT)0.38268343236508977173;
  const RT r2 = (RT)0.70710678118654752440;
  RT x, y;
  switch (m) {
    case 0: x = RT(1); y = RT(0); break;
    case 1: x = c1; y = -s1; break;
    case 2: x = r2; y = -r2; break;
    case 3: x = s1; y = -c1; break;
    case 4: x = RT(0); y = RT(-1); break;
    case 6: x = -r2; y = -r2; break;
    default: x = -c1; y = s1; break;  // m = 9
  }
  return mkc<CT>(x, inv ? -y : y);
}

// in-place 16-point DFT: v[a] -> V[k], both in natural order
template <class CT>
__device__ __forceinline__ void dft16(CT (&v)[16], bool inv) {
  CT t[16];  // t[a1 + 4 e0]
#pragma unroll
  for (int a1 = 0; a1 < 4; ++a1) {
    CT q[4] = {v[a1], v[a1 + 4], v[a1 + 8], v[a1 + 12]};
    DftSmall<4, CT>::run(q, inv);
#pragma unroll
    for (int e0 = 0; e0 < 4; ++e0)
      t[a1 + 4 * e0] = (a1 * e0 == 0) ? q[e0] : cmul(q[e0], w16<CT>(a1 * e0, inv));
  }
#pragma unroll
  for (int e0 = 0; e0 < 4; ++e0) {
    CT q[4] = {t[4 * e0], t[4 * e0 + 1], t[4 * e0 + 2], t[4 * e0 + 3]};
    DftSmall<4, CT>::run(q, inv);
#pragma unroll
    for (int e1 = 0; e1 < 4; ++e1) v[e0 + 4 * e1] = q[e1];
  }
}

// the inner half of the transform on thread b: DFT over a, then W256^(bc)
template <class CT>
__device__ __forceinline__ void fft256_inner(CT (&v)[16], int b, const CT* __restrict__ tw,
                                             bool inv) {
  dft16(v, inv);
#pragma unroll
  for (int c = 1; c < 16; ++c) {
    CT w = __ldg(tw + b * c);
    if (inv) w.y = -w.y;
    v[c] = cmul(v[c], w);
  }
}

}  // namespace nse
