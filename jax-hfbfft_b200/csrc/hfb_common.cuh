// Shared device building blocks for the HF-BCS kernels (sm_100a).
//
//  * complex arithmetic on float2 / double2 (interleaved re,im = the memory
//    layout of torch.complex64 / complex128 and of the reference's complex128
//    psi[nst, 2, nx, ny, nz]),
//  * compile-time twiddle factors (Taylor series evaluated by the compiler),
//  * register-resident DFT codelets of small size,
//  * the cooperative "pencil" FFT: P threads own one length-N line, each
//    holding M = N/P points at stride P; one shared-memory transpose per
//    transform (four-step Cooley-Tukey, N = P * M).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace hfb {

// ----------------------------------------------------------------- complex --
template <class R> struct C2;
template <> struct C2<float> { using T = float2; };
template <> struct C2<double> { using T = double2; };
template <class R> using cplx = typename C2<R>::T;

template <class R> __host__ __device__ __forceinline__ cplx<R> mk(R a, R b) { cplx<R> z; z.x = a; z.y = b; return z; }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

template <class Z> __device__ __forceinline__ Z cmul(Z a, Z b) { Z r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r; }
// conj(a) * b
template <class Z> __device__ __forceinline__ Z cmulc(Z a, Z b) { Z r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r; }
// i * a
template <class Z> __device__ __forceinline__ Z mul_i(Z a) { Z r; r.x = -a.y; r.y = a.x; return r; }
// (re + i im) * a  with real re, im
template <class Z, class R> __device__ __forceinline__ Z cmulri(R re, R im, Z a) { Z r; r.x = re * a.x - im * a.y; r.y = re * a.y + im * a.x; return r; }
template <class Z> __device__ __forceinline__ Z czero() { Z r; r.x = 0; r.y = 0; return r; }

// --------------------------------------------------- compile-time twiddles --
// cos / sin of 2*pi*j/m evaluated at compile time: exact octant reduction,
// then a Taylor series on [0, pi/4] (terms to x^27; error below 1e-17).
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int k = 1; k < 14; ++k) { t = -t * x * x / ((2.0 * k) * (2.0 * k + 1.0)); s += t; }
  return s;
}
constexpr double taylor_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int k = 1; k < 14; ++k) { t = -t * x * x / ((2.0 * k - 1.0) * (2.0 * k)); s += t; }
  return s;
}
// angle = 2*pi * j / m, j reduced into [0, m)
constexpr double tw_cos_sin(long j, long m, bool want_sin) {
  j %= m; if (j < 0) j += m;
  // work in units of 1/(8m) turns: a = 8*j in [0, 8m)
  long a = 8 * j;
  long oct = a / m;              // octant 0..7
  long rem = a - oct * m;        // position inside octant, in units of 1/(8m) turn
  // theta = (oct * m + rem) / (8m) * 2pi ; within-octant angle phi = rem/(8m)*2pi in [0, pi/4)
  double phi = (double)rem * (2.0 * kPi) / (8.0 * (double)m);
  double psi = (double)(m - rem) * (2.0 * kPi) / (8.0 * (double)m);  // pi/4 - phi
  double c = 0, s = 0;
  switch (oct) {
    case 0: c = taylor_cos(phi); s = taylor_sin(phi); break;
    case 1: c = taylor_sin(psi); s = taylor_cos(psi); break;
    case 2: c = -taylor_sin(phi); s = taylor_cos(phi); break;
    case 3: c = -taylor_cos(psi); s = taylor_sin(psi); break;
    case 4: c = -taylor_cos(phi); s = -taylor_sin(phi); break;
    case 5: c = -taylor_sin(psi); s = -taylor_cos(psi); break;
    case 6: c = taylor_sin(phi); s = -taylor_cos(phi); break;
    default: c = taylor_cos(psi); s = -taylor_sin(psi); break;
  }
  return want_sin ? s : c;
}

// x * w_m^(e) with w_m = exp(SIGN * 2 pi i / m); SIGN = -1 forward, +1 inverse.
template <int SIGN, long E, long MM, class Z>
__device__ __forceinline__ Z twiddle_const(Z x) {
  constexpr long e = ((E % MM) + MM) % MM;
  if constexpr (e == 0) {
    return x;
  } else if constexpr (4 * e == MM) {          // quarter turn
    Z r; if (SIGN < 0) { r.x = x.y; r.y = -x.x; } else { r.x = -x.y; r.y = x.x; } return r;
  } else if constexpr (2 * e == MM) {          // half turn
    Z r; r.x = -x.x; r.y = -x.y; return r;
  } else if constexpr (4 * e == 3 * MM) {      // three quarters
    Z r; if (SIGN < 0) { r.x = -x.y; r.y = x.x; } else { r.x = x.y; r.y = -x.x; } return r;
  } else {
    constexpr double c = tw_cos_sin(e, MM, false);
    constexpr double s = (SIGN < 0 ? -1.0 : 1.0) * tw_cos_sin(e, MM, true);
    using R = decltype(x.x);
    Z r; r.x = (R)c * x.x - (R)s * x.y; r.y = (R)c * x.y + (R)s * x.x; return r;
  }
}

// ------------------------------------------------------------- codelets --
// In-place DFT of length M held in registers: X[k] = sum_j x[j] w^(jk),
// w = exp(SIGN 2 pi i / M).  Composite sizes split M = A * B (A the smallest
// factor): j = a + A b, k = k2 + B k1.
template <int M> struct small_factor {
  static constexpr int value = (M % 4 == 0 && M != 4 && M != 8) ? 4 : (M % 2 == 0 ? 2 : (M % 3 == 0 ? 3 : (M % 5 == 0 ? 5 : M)));
};

template <int M, int SIGN, class Z> struct DFT;

template <int SIGN, class Z> struct DFT<1, SIGN, Z> { __device__ __forceinline__ static void run(Z*) {} };
template <int SIGN, class Z> struct DFT<2, SIGN, Z> {
  __device__ __forceinline__ static void run(Z* x) { Z a = x[0], b = x[1]; x[0] = a + b; x[1] = a - b; }
};
template <int SIGN, class Z> struct DFT<4, SIGN, Z> {
  __device__ __forceinline__ static void run(Z* x) {
    Z t0 = x[0] + x[2], t1 = x[0] - x[2], t2 = x[1] + x[3], t3 = x[1] - x[3];
    t3 = twiddle_const<SIGN, 1, 4>(t3);
    x[0] = t0 + t2; x[2] = t0 - t2; x[1] = t1 + t3; x[3] = t1 - t3;
  }
};
template <int SIGN, class Z> struct DFT<3, SIGN, Z> {
  __device__ __forceinline__ static void run(Z* x) {
    using R = decltype(x[0].x);
    constexpr R h = (R)0.5;
    constexpr R s3 = (R)(SIGN * 0.86602540378443864676372317075293618);
    Z a = x[0], b = x[1], c = x[2];
    Z sum = b + c, dif = b - c;
    Z m; m.x = a.x - h * sum.x; m.y = a.y - h * sum.y;
    Z r; r.x = -s3 * dif.y; r.y = s3 * dif.x;     // SIGN*i*sqrt(3)/2 * (b - c)
    x[0] = a + sum; x[1] = m + r; x[2] = m - r;
  }
};
template <int SIGN, class Z> struct DFT<5, SIGN, Z> {
  __device__ __forceinline__ static void run(Z* x) {
    using R = decltype(x[0].x);
    constexpr R c1 = (R)0.30901699437494742410229341718281906;   // cos(2pi/5)
    constexpr R c2 = (R)-0.80901699437494742410229341718281906;  // cos(4pi/5)
    constexpr R s1 = (R)(SIGN * 0.95105651629515357211643933337938214);  // sin(2pi/5)
    constexpr R s2 = (R)(SIGN * 0.58778525229247312916870595463907277);  // sin(4pi/5)
    Z a = x[0];
    Z p1 = x[1] + x[4], m1 = x[1] - x[4], p2 = x[2] + x[3], m2 = x[2] - x[3];
    Z u1, u2, v1, v2;
    u1.x = a.x + c1 * p1.x + c2 * p2.x; u1.y = a.y + c1 * p1.y + c2 * p2.y;
    u2.x = a.x + c2 * p1.x + c1 * p2.x; u2.y = a.y + c2 * p1.y + c1 * p2.y;
    // i*(s1*m1 + s2*m2) and i*(s2*m1 - s1*m2)
    v1.x = -(s1 * m1.y + s2 * m2.y); v1.y = s1 * m1.x + s2 * m2.x;
    v2.x = -(s2 * m1.y - s1 * m2.y); v2.y = s2 * m1.x - s1 * m2.x;
    x[0] = a + p1 + p2;
    x[1] = u1 + v1; x[4] = u1 - v1;
    x[2] = u2 + v2; x[3] = u2 - v2;
  }
};

template <int M, int SIGN, class Z> struct DFT {
  static constexpr int A = small_factor<M>::value;
  static constexpr int B = M / A;
  static_assert(A * B == M && A > 1 && B > 1, "unsupported DFT size");
  template <int a> __device__ __forceinline__ static void inner(Z* x, Z (&t)[A][B]) {
    if constexpr (a < A) {
#pragma unroll
      for (int b = 0; b < B; ++b) t[a][b] = x[a + A * b];
      DFT<B, SIGN, Z>::run(t[a]);
      twid<a, 0>(t);
      inner<a + 1>(x, t);
    }
  }
  template <int a, int k2> __device__ __forceinline__ static void twid(Z (&t)[A][B]) {
    if constexpr (k2 < B) { t[a][k2] = twiddle_const<SIGN, (long)a * k2, M>(t[a][k2]); twid<a, k2 + 1>(t); }
  }
  __device__ __forceinline__ static void run(Z* x) {
    Z t[A][B];
    inner<0>(x, t);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) {
      Z u[A];
#pragma unroll
      for (int a = 0; a < A; ++a) u[a] = t[a][k2];
      DFT<A, SIGN, Z>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) x[k2 + B * k1] = u[k1];
    }
  }
};

// ------------------------------------------------------------ pencil FFT --
// Line of length N split over P cooperating lanes (consecutive lanes of one
// warp).  Lane p owns x[p + P m], m = 0..M-1 in the "space" distribution.
// After forward(), lane q owns X[k2 + M k1] for k2 = q + P t (t < T, k2 < M)
// and k1 = 0..P-1 in f[t][k1] (the "frequency" distribution); inverse() takes
// that distribution back to the space distribution.  Unnormalised in both
// directions.  ``xb`` is this line's shared exchange buffer (N elements) and
// ``tw`` a shared table tw[j] = exp(-2 pi i j / N).
template <class R, int N_, int P_> struct Pencil {
  static constexpr int N = N_;
  static constexpr int P = P_;
  static constexpr int M = N / P;
  static constexpr int T = (M + P - 1) / P;
  static_assert(N % P == 0 && 32 % P == 0, "pencil split");
  using Z = cplx<R>;

  // Index of frequency slot (t, k1) held by lane q.
  __device__ __forceinline__ static int freq(int q, int t, int k1) { return q + P * t + M * k1; }
  __device__ __forceinline__ static bool valid(int q, int t) { return q + P * t < M; }

  // e = p k2 with p < P and k2 < M at every call, so e <= (P - 1)(M - 1) < N
  template <int SIGN>
  __device__ __forceinline__ static Z tw_mul(Z x, const Z* tw, int e) {
    Z w = tw[e];
    if (SIGN > 0) w.y = -w.y;
    return cmul(x, w);
  }

  __device__ __forceinline__ static void forward(Z (&v)[M], Z (&f)[T][P], Z* xb, const Z* tw, int p, unsigned mask) {
    DFT<M, -1, Z>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < M; ++k2) xb[k2 * P + p] = (k2 == 0 || p == 0) ? v[k2] : tw_mul<-1>(v[k2], tw, p * k2);
    __syncwarp(mask);
#pragma unroll
    for (int t = 0; t < T; ++t) {
      int k2 = p + P * t;
      if (T * P == M || k2 < M) {
#pragma unroll
        for (int pp = 0; pp < P; ++pp) f[t][pp] = xb[k2 * P + pp];
        DFT<P, -1, Z>::run(f[t]);
      }
    }
    __syncwarp(mask);
  }

  __device__ __forceinline__ static void inverse(Z (&f)[T][P], Z (&v)[M], Z* xb, const Z* tw, int p, unsigned mask) {
#pragma unroll
    for (int t = 0; t < T; ++t) {
      int k2 = p + P * t;
      if (T * P == M || k2 < M) {
        DFT<P, +1, Z>::run(f[t]);
#pragma unroll
        for (int pp = 0; pp < P; ++pp) xb[k2 * P + pp] = (k2 == 0 || pp == 0) ? f[t][pp] : tw_mul<+1>(f[t][pp], tw, pp * k2);
      }
    }
    __syncwarp(mask);
#pragma unroll
    for (int k2 = 0; k2 < M; ++k2) v[k2] = xb[k2 * P + p];
    DFT<M, +1, Z>::run(v);
    __syncwarp(mask);
  }
};

// Pencil split (P lanes per line) for each supported length; double
// precision uses more lanes per line to keep the register footprint down.
template <class R, int N> struct PencilSplit {
  static constexpr int P = sizeof(R) == 8 ? ((N >= 32) ? 8 : (N >= 16 ? 4 : 2))
                                          : ((N >= 64) ? 8 : (N >= 16 ? 4 : 2));
};

// Fill a shared twiddle table tw[j] = exp(-2 pi i j / N), j < N (double
// precision sincospi, rounded to R).
template <class R>
__device__ __forceinline__ void fill_twiddles(cplx<R>* tw, int n) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)j / (double)n, &s, &c);
    tw[j] = mk<R>((R)c, (R)s);
  }
}

// Signed wave number of FFT bin k for length n (bin n/2 maps to n/2).
__device__ __forceinline__ int signed_k(int k, int n) { return k <= n / 2 ? k : k - n; }

}  // namespace hfb
