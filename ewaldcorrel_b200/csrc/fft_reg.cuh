// Register-resident DFTs of compile-time length R (1..16 and composites of
// them) and the helpers of the two-level line transform.
//
// dft<R, SIGN>(v) computes X[k] = sum_j v[j] exp(SIGN 2 pi i j k / R) in
// place, input and output in natural order, entirely in registers:
//   R = 2, 3, 4          written-out butterflies;
//   R odd prime          direct DFT with the (j, R - j) symmetric pairing;
//   R composite          R = A * B four-step: B DFTs of length A on the
//                        stride-B subsequences, twiddles W_R^(j2 k1), A DFTs
//                        of length B, all indices compile-time constants.
// Twiddle constants cos/sin(2 pi k / R) are evaluated at compile time by a
// Taylor series on the octant-reduced angle (|x| <= pi/4, 14 terms: error
// below 1e-17), so no table or transcendental runs at run time.
//
// A line of length n = n1 * n2 is transformed in two register steps with one
// exchange between them (the four-step decomposition):
//   X[k1 + n1 k2] = sum_j2 W_n2^(j2 k2) W_n^(j2 k1) sum_j1 x[j2 + n2 j1] W_n1^(j1 k1)
// step 1: task j2 loads x[j2 + n2 j1] (j1 < n1), dft<n1>, multiplies by
//         W_n^(j2 k1), stores to the exchange buffer;
// step 2: task k1 loads the n2 values of its k1, dft<n2>, holding
//         X[k1 + n1 k2] for all k2.
// The inverse runs the same steps backwards (dft<n2> on the held values,
// conjugate twiddles, exchange, dft<n1>), returning the line to the task
// layout of step 1.  Everything is __host__ __device__ so the arithmetic can
// be checked against a direct DFT on the CPU.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace spme {
namespace rdft {

#define RD_HD __host__ __device__ __forceinline__

constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double sin_poly(double x) {
  double t = x, s = x;
  for (int i = 1; i < 14; i++) {
    t *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    s += t;
  }
  return s;
}
constexpr double cos_poly(double x) {
  double t = 1.0, s = 1.0;
  for (int i = 1; i < 14; i++) {
    t *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    s += t;
  }
  return s;
}
// cos(2 pi k / R): the octant comes from the integer ratio, the remainder
// angle lies in [0, pi/4).
constexpr double cos2pi(long k, long R) {
  k %= R;
  if (k < 0) k += R;
  const long o = (8 * k) / R;
  const double x = 2.0 * kPi * ((double)(8 * k - o * R) / (8.0 * (double)R));
  switch (o) {
    case 0: return cos_poly(x);
    case 1: return sin_poly(kPi / 4 - x);
    case 2: return -sin_poly(x);
    case 3: return -cos_poly(kPi / 4 - x);
    case 4: return -cos_poly(x);
    case 5: return -sin_poly(kPi / 4 - x);
    case 6: return sin_poly(x);
    default: return cos_poly(kPi / 4 - x);
  }
}
// sin(t) = cos(t - pi/2): 2 pi k / R - pi/2 = 2 pi (4k - R) / (4R)
constexpr double sin2pi(long k, long R) { return cos2pi(4 * k - R, 4 * R); }

constexpr bool is_prime(int r) {
  if (r < 2) return false;
  for (int p = 2; p * p <= r; p++)
    if (r % p == 0) return false;
  return true;
}
// First factor of a composite length: 4 when it divides (radix-4 inner
// butterflies need no multiplies), else the smallest prime factor.
constexpr int split_factor(int r) {
  if (r % 4 == 0 && r > 4) return 4;
  for (int p = 2; p < r; p++)
    if (r % p == 0) return p;
  return r;
}

#pragma nv_exec_check_disable
template <int B, int E, class F>
RD_HD void sfor(F &&f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

RD_HD float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
RD_HD float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// SIGN * i * a
template <int SIGN>
RD_HD float2 rot(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
// a * W_R^K with W_R = exp(SIGN 2 pi i / R), K a compile-time constant
template <int R, int SIGN, int K>
RD_HD float2 mul_w(float2 a) {
  constexpr int k = ((K % R) + R) % R;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (2 * k == R) {
    return make_float2(-a.x, -a.y);
  } else if constexpr (4 * k == R) {
    return rot<SIGN>(a);
  } else if constexpr (4 * k == 3 * R) {
    return rot<-SIGN>(a);
  } else if constexpr (8 * k == R || 8 * k == 3 * R || 8 * k == 5 * R || 8 * k == 7 * R) {
    constexpr float h = 0.70710678118654752440f;
    constexpr float c = (float)cos2pi(k, R), s = (float)(SIGN * sin2pi(k, R));
    // c, s = +-h
    return make_float2(h * ((c > 0 ? a.x : -a.x) - (s > 0 ? a.y : -a.y)),
                       h * ((s > 0 ? a.x : -a.x) + (c > 0 ? a.y : -a.y)));
  } else {
    constexpr float c = (float)cos2pi(k, R), s = (float)(SIGN * sin2pi(k, R));
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

template <int R, int SIGN>
RD_HD void dft(float2 (&v)[R]);

// Odd prime R: X[k] = v0 + sum_j a_j cos(2 pi j k / R) + SIGN i sum_j b_j sin(2 pi j k / R),
// a_j = v_j + v_{R-j}, b_j = v_j - v_{R-j}; X[R-k] flips the sine part.
template <int R, int SIGN>
RD_HD void dft_prime(float2 (&v)[R]) {
  constexpr int H = (R - 1) / 2;
  float2 a[H], b[H];
  float2 s0 = v[0];
  sfor<1, H + 1>([&](auto J) {
    constexpr int j = decltype(J)::value;
    a[j - 1] = add(v[j], v[R - j]);
    b[j - 1] = sub(v[j], v[R - j]);
    s0 = add(s0, a[j - 1]);
  });
  float2 out[R];
  out[0] = s0;
  sfor<1, H + 1>([&](auto K) {
    constexpr int k = decltype(K)::value;
    float2 re = v[0], im = make_float2(0.f, 0.f);
    sfor<1, H + 1>([&](auto J) {
      constexpr int j = decltype(J)::value;
      constexpr float c = (float)cos2pi((long)j * k, R), s = (float)sin2pi((long)j * k, R);
      re.x = fmaf(a[j - 1].x, c, re.x);
      re.y = fmaf(a[j - 1].y, c, re.y);
      im.x = fmaf(b[j - 1].x, s, im.x);
      im.y = fmaf(b[j - 1].y, s, im.y);
    });
    const float2 r = rot<SIGN>(im);
    out[k] = add(re, r);
    out[R - k] = sub(re, r);
  });
  sfor<0, R>([&](auto K) {
    constexpr int k = decltype(K)::value;
    v[k] = out[k];
  });
}

template <int R, int SIGN>
RD_HD void dft_composite(float2 (&v)[R]) {
  constexpr int A = split_factor(R), B = R / A;
  float2 t[B][A];
  sfor<0, B>([&](auto J2) {
    constexpr int j2 = decltype(J2)::value;
    float2 u[A];
    sfor<0, A>([&](auto J1) {
      constexpr int j1 = decltype(J1)::value;
      u[j1] = v[j2 + B * j1];
    });
    dft<A, SIGN>(u);
    sfor<0, A>([&](auto K1) {
      constexpr int k1 = decltype(K1)::value;
      t[j2][k1] = mul_w<R, SIGN, j2 * k1>(u[k1]);
    });
  });
  sfor<0, A>([&](auto K1) {
    constexpr int k1 = decltype(K1)::value;
    float2 w[B];
    sfor<0, B>([&](auto J2) {
      constexpr int j2 = decltype(J2)::value;
      w[j2] = t[j2][k1];
    });
    dft<B, SIGN>(w);
    sfor<0, B>([&](auto K2) {
      constexpr int k2 = decltype(K2)::value;
      v[k1 + A * k2] = w[k2];
    });
  });
}

template <int R, int SIGN>
RD_HD void dft(float2 (&v)[R]) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = add(a, b);
    v[1] = sub(a, b);
  } else if constexpr (R == 3) {
    constexpr float s = 0.86602540378443864676f;
    const float2 t = add(v[1], v[2]), d = sub(v[1], v[2]);
    const float2 mid = make_float2(fmaf(-0.5f, t.x, v[0].x), fmaf(-0.5f, t.y, v[0].y));
    const float2 r = rot<SIGN>(make_float2(s * d.x, s * d.y));
    v[0] = add(v[0], t);
    v[1] = add(mid, r);
    v[2] = sub(mid, r);
  } else if constexpr (R == 4) {
    const float2 t0 = add(v[0], v[2]), t1 = sub(v[0], v[2]);
    const float2 t2 = add(v[1], v[3]), t3 = rot<SIGN>(sub(v[1], v[3]));
    v[0] = add(t0, t2);
    v[2] = sub(t0, t2);
    v[1] = add(t1, t3);
    v[3] = sub(t1, t3);
  } else if constexpr (is_prime(R)) {
    dft_prime<R, SIGN>(v);
  } else {
    dft_composite<R, SIGN>(v);
  }
}

// Largest register length handled by the two-level line transform.
constexpr int kMaxRadix = 16;

// Calls f(std::integral_constant<int, R>) for a run-time R in [1, kMaxRadix];
// returns false for any other R.
#pragma nv_exec_check_disable
template <class F>
RD_HD bool with_radix(int r, F &&f) {
  switch (r) {
    case 1: f(std::integral_constant<int, 1>{}); return true;
    case 2: f(std::integral_constant<int, 2>{}); return true;
    case 3: f(std::integral_constant<int, 3>{}); return true;
    case 4: f(std::integral_constant<int, 4>{}); return true;
    case 5: f(std::integral_constant<int, 5>{}); return true;
    case 6: f(std::integral_constant<int, 6>{}); return true;
    case 7: f(std::integral_constant<int, 7>{}); return true;
    case 8: f(std::integral_constant<int, 8>{}); return true;
    case 9: f(std::integral_constant<int, 9>{}); return true;
    case 10: f(std::integral_constant<int, 10>{}); return true;
    case 11: f(std::integral_constant<int, 11>{}); return true;
    case 12: f(std::integral_constant<int, 12>{}); return true;
    case 13: f(std::integral_constant<int, 13>{}); return true;
    case 14: f(std::integral_constant<int, 14>{}); return true;
    case 15: f(std::integral_constant<int, 15>{}); return true;
    case 16: f(std::integral_constant<int, 16>{}); return true;
    default: return false;
  }
}

// n = n1 * n2 with both factors <= kMaxRadix, balanced (n1 >= n2, n1 as
// small as possible).  Returns false when n has no such split.
inline bool split_line(int n, int &n1, int &n2) {
  for (int a = 1; a <= kMaxRadix; a++) {
    if (n % a) continue;
    const int b = n / a;
    if (b <= kMaxRadix && b <= a) {
      n1 = a;
      n2 = b;
      return true;
    }
  }
  return false;
}

#undef RD_HD

}  // namespace rdft
}  // namespace spme
