// In-shared-memory mixed-radix Stockham FFT executed by a group of threads.
//
// This replaces the role cuFFT plays in the reference (cufftPlanMany /
// cufftExecR2C / cufftExecC2R at sporco_cuda/src/cbpdn.cu:171-180, 283-350):
// every 1-D transform of the ADMM iteration (length W along image rows,
// length H along columns) is done by one thread group inside a fused kernel,
// on data staged in shared memory, so that the transforms never make their
// own round trip through HBM.
//
// Conventions
//  * Forward transform, unnormalised: X[k] = sum_j x[j] exp(-2 pi i jk/n)
//    (numpy / cuFFT convention).  Inverse transforms are done by the callers
//    as conj(FFT(conj(x))), which costs nothing extra because the callers
//    stage the data into and out of shared memory anyway.
//  * Twiddles: one table tw[j] = exp(-2 pi i j/n), j < n, evaluated in
//    double precision and rounded to float.  Every twiddle of every
//    pass is an entry of that table.
//  * Stockham auto-sort (natural order in and out): a pass of radix R with
//    Ns = product of the previous radices maps butterfly j (0 <= j < n/R)
//        in[j + q n/R] (q < R)  ->  out[(j/Ns) Ns R + j%Ns + q Ns]
//    after multiplying input q by w_{Ns R}^{q (j%Ns)} and taking an R-point
//    DFT.  Passes are done in place: every thread first loads and combines
//    all of its butterflies into registers, the group synchronises, then all
//    results are stored.
//  * A group of g threads does one transform; several groups of a CTA run
//    transforms of the same length in lock step and synchronise with
//    __syncthreads() (all groups must call the routine together).
//  * The n elements of a transform may be strided (element i at data[i*st]),
//    so that several transforms can be interleaved in shared memory exactly
//    as their columns are interleaved in global memory.
//  * MAXE bounds the elements one thread holds: the caller guarantees
//    n <= MAXE * g.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define SC_FFT_MAX_PASS 24

struct FftPlan {
  int n;
  int npass;
  int radix[SC_FFT_MAX_PASS];
};

// ---------------------------------------------------------------- complex --
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// (-i) * a
__device__ __forceinline__ float2 c_mul_mi(float2 a) { return make_float2(a.y, -a.x); }
// (+i) * a
__device__ __forceinline__ float2 c_mul_pi(float2 a) { return make_float2(-a.y, a.x); }
__device__ __forceinline__ float c_abs2(float2 a) { return a.x * a.x + a.y * a.y; }

// ------------------------------------------------------------- butterflies --
// Forward R-point DFTs, in registers.  Constants are exact values of the
// roots of unity (cos/sin of 2 pi/3, 2 pi/5, 4 pi/5, pi/4) to float precision.
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0];
  v[0] = c_add(a, v[1]);
  v[1] = c_sub(a, v[1]);
}

__device__ __forceinline__ void dft3(float2* v) {
  const float h = 0.8660254037844386f;  // sin(2 pi / 3)
  float2 s = c_add(v[1], v[2]);
  float2 d = c_sub(v[1], v[2]);
  float2 a = v[0];
  v[0] = c_add(a, s);
  float2 m = make_float2(a.x - 0.5f * s.x, a.y - 0.5f * s.y);
  float2 t = c_mul_mi(c_scale(d, h));  // -i sin(2pi/3) (b - c)
  v[1] = c_add(m, t);
  v[2] = c_sub(m, t);
}

__device__ __forceinline__ void dft4(float2* v) {
  float2 t0 = c_add(v[0], v[2]);
  float2 t1 = c_sub(v[0], v[2]);
  float2 t2 = c_add(v[1], v[3]);
  float2 t3 = c_mul_mi(c_sub(v[1], v[3]));
  v[0] = c_add(t0, t2);
  v[2] = c_sub(t0, t2);
  v[1] = c_add(t1, t3);
  v[3] = c_sub(t1, t3);
}

__device__ __forceinline__ void dft5(float2* v) {
  const float c1 = 0.30901699437494745f;   // cos(2 pi/5)
  const float c2 = -0.8090169943749475f;   // cos(4 pi/5)
  const float s1 = 0.9510565162951535f;    // sin(2 pi/5)
  const float s2 = 0.5877852522924731f;    // sin(4 pi/5)
  float2 a0 = v[0];
  float2 t1 = c_add(v[1], v[4]), d1 = c_sub(v[1], v[4]);
  float2 t2 = c_add(v[2], v[3]), d2 = c_sub(v[2], v[3]);
  v[0] = c_add(a0, c_add(t1, t2));
  float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
  float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
  float2 e1 = c_mul_mi(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
  float2 e2 = c_mul_mi(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
  v[1] = c_add(m1, e1);
  v[4] = c_sub(m1, e1);
  v[2] = c_add(m2, e2);
  v[3] = c_sub(m2, e2);
}

__device__ __forceinline__ void dft8(float2* v) {
  const float r = 0.7071067811865476f;  // cos(pi/4)
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e);
  dft4(o);
  // w8^1 = r (1 - i), w8^2 = -i, w8^3 = r (-1 - i)
  float2 o1 = make_float2(r * (o[1].x + o[1].y), r * (o[1].y - o[1].x));
  float2 o2 = c_mul_mi(o[2]);
  float2 o3 = make_float2(r * (o[3].y - o[3].x), -r * (o[3].x + o[3].y));
  v[0] = c_add(e[0], o[0]);
  v[4] = c_sub(e[0], o[0]);
  v[1] = c_add(e[1], o1);
  v[5] = c_sub(e[1], o1);
  v[2] = c_add(e[2], o2);
  v[6] = c_sub(e[2], o2);
  v[3] = c_add(e[3], o3);
  v[7] = c_sub(e[3], o3);
}

// 16-point DFT as 4 x 4: DFT4 over the stride-4 subsequences, twiddles
// w16^(n2 k1), DFT4 across them (X[k1 + 4 k2]).
__device__ __forceinline__ void dft16(float2* v) {
  const float c1 = 0.9238795325112867f;  // cos(pi/8)
  const float s1 = 0.3826834323650898f;  // sin(pi/8)
  const float r = 0.7071067811865476f;   // cos(pi/4)
  float2 y[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    float2 a[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
    dft4(a);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = a[k1];
  }
  // w16^1 = (c1, -s1), w16^2 = (r, -r), w16^3 = (s1, -c1), w16^4 = -i,
  // w16^6 = (-r, -r), w16^9 = (-c1, s1)
  y[1][1] = c_mul(y[1][1], make_float2(c1, -s1));
  y[1][2] = c_mul(y[1][2], make_float2(r, -r));
  y[1][3] = c_mul(y[1][3], make_float2(s1, -c1));
  y[2][1] = c_mul(y[2][1], make_float2(r, -r));
  y[2][2] = c_mul_mi(y[2][2]);
  y[2][3] = c_mul(y[2][3], make_float2(-r, -r));
  y[3][1] = c_mul(y[3][1], make_float2(s1, -c1));
  y[3][2] = c_mul(y[3][2], make_float2(-r, -r));
  y[3][3] = c_mul(y[3][3], make_float2(-c1, s1));
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    float2 b[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
    dft4(b);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
  }
}

template <int R>
__device__ __forceinline__ void dft_r(float2* v) {
  if constexpr (R == 2) dft2(v);
  else if constexpr (R == 3) dft3(v);
  else if constexpr (R == 4) dft4(v);
  else if constexpr (R == 5) dft5(v);
  else if constexpr (R == 8) dft8(v);
  else if constexpr (R == 16) dft16(v);
}

// Multiply v[q] (q = 1..R-1) by w^q, w = tw[i1]: w, w^4 and w^8 come from the
// table, the other powers are products of at most two factors.
template <int R>
__device__ __forceinline__ void twiddle_r(float2* v, const float2* __restrict__ tw, int i1) {
  const float2 w1 = __ldg(&tw[i1]);
  if constexpr (R == 2) {
    v[1] = c_mul(v[1], w1);
  } else if constexpr (R == 3) {
    v[1] = c_mul(v[1], w1);
    v[2] = c_mul(v[2], c_mul(w1, w1));
  } else {
    const float2 w2 = c_mul(w1, w1);
    const float2 w3 = c_mul(w2, w1);
    v[1] = c_mul(v[1], w1);
    v[2] = c_mul(v[2], w2);
    v[3] = c_mul(v[3], w3);
    if constexpr (R == 5) {
      v[4] = c_mul(v[4], c_mul(w2, w2));
    } else if constexpr (R >= 8) {
      const float2 w4 = __ldg(&tw[4 * i1]);
      v[4] = c_mul(v[4], w4);
#pragma unroll
      for (int q = 1; q < 4; ++q) v[4 + q] = c_mul(v[4 + q], c_mul(w4, q == 1 ? w1 : q == 2 ? w2 : w3));
      if constexpr (R == 16) {
        const float2 w8 = __ldg(&tw[8 * i1]);
        const float2 w12 = c_mul(w8, w4);
        v[8] = c_mul(v[8], w8);
        v[12] = c_mul(v[12], w12);
#pragma unroll
        for (int q = 1; q < 4; ++q) {
          const float2 wq = q == 1 ? w1 : q == 2 ? w2 : w3;
          v[8 + q] = c_mul(v[8 + q], c_mul(w8, wq));
          v[12 + q] = c_mul(v[12 + q], c_mul(w12, wq));
        }
      }
    }
  }
}

// ------------------------------------------------------------------ passes --
template <int R, int MAXE>
__device__ __forceinline__ void stockham_pass(float2* data, int n, int Ns, int st,
                                              const float2* __restrict__ tw,
                                              int t, int g) {
  constexpr int MAXB = (MAXE + R - 1) / R;
  const int B = n / R;
  const int step = n / (Ns * R);
  float2 v[MAXB][R];
#pragma unroll
  for (int i = 0; i < MAXB; ++i) {
    const int j = t + i * g;
    if (j < B) {
#pragma unroll
      for (int q = 0; q < R; ++q) v[i][q] = data[(j + q * B) * st];
      if (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int q = 1; q < R; ++q) v[i][q] = c_mul(v[i][q], __ldg(&tw[q * k * step]));
      }
      dft_r<R>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MAXB; ++i) {
    const int j = t + i * g;
    if (j < B) {
      const int k = j % Ns;
      const int base = (j - k) * R + k;
#pragma unroll
      for (int q = 0; q < R; ++q) data[(base + q * Ns) * st] = v[i][q];
    }
  }
  __syncthreads();
}

// Any radix (used for prime factors other than 2, 3, 5): each thread
// computes whole outputs, O(R) work per output.
template <int MAXE>
__device__ __noinline__ void generic_pass(float2* data, int n, int R, int Ns, int st,
                                          const float2* __restrict__ tw, int t, int g) {
  const int B = n / R;
  const int step = n / (Ns * R);
  float2 out[MAXE];
#pragma unroll
  for (int i = 0; i < MAXE; ++i) {
    const int o = t + i * g;
    if (o < n) {
      const int q = o / B;
      const int j = o - q * B;
      const int k = j % Ns;
      const int e1 = k * step + q * B;  // < n
      float2 acc = make_float2(0.f, 0.f);
      int e = 0;
      for (int s = 0; s < R; ++s) {
        const float2 x = data[(j + s * B) * st];
        const float2 w = __ldg(&tw[e]);
        acc.x += x.x * w.x - x.y * w.y;
        acc.y += x.x * w.y + x.y * w.x;
        e += e1;
        if (e >= n) e -= n;
      }
      out[i] = acc;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MAXE; ++i) {
    const int o = t + i * g;
    if (o < n) {
      const int q = o / B;
      const int j = o - q * B;
      const int k = j % Ns;
      data[((j - k) * R + k + q * Ns) * st] = out[i];
    }
  }
  __syncthreads();
}

// One pass of a runtime plan.  Kept out of line: with the passes inlined into
// a loop over a runtime radix sequence the register allocation of the
// calling kernel grows past 200 registers.
template <int MAXE>
__device__ __noinline__ void fft_pass(float2* data, int n, int R, int Ns, int st,
                                      const float2* __restrict__ tw, int t, int g) {
  switch (R) {
    case 2: stockham_pass<2, MAXE>(data, n, Ns, st, tw, t, g); break;
    case 3: stockham_pass<3, MAXE>(data, n, Ns, st, tw, t, g); break;
    case 4: stockham_pass<4, MAXE>(data, n, Ns, st, tw, t, g); break;
    case 5: stockham_pass<5, MAXE>(data, n, Ns, st, tw, t, g); break;
    case 8: stockham_pass<8, MAXE>(data, n, Ns, st, tw, t, g); break;
    default: generic_pass<MAXE>(data, n, R, Ns, st, tw, t, g); break;
  }
}

// In-place forward DFT of data[0], data[st], ..., data[(n-1) st] (shared
// memory) by a group of g threads, for any n (runtime plan; the fallback).
template <int MAXE>
__device__ __forceinline__ void fft_forward(float2* data, const FftPlan& P, int st,
                                            const float2* __restrict__ tw, int t, int g) {
  int Ns = 1;
  const int np = P.npass;
  for (int p = 0; p < np; ++p) {
    const int R = P.radix[p];
    fft_pass<MAXE>(data, P.n, R, Ns, st, tw, t, g);
    Ns *= R;
  }
}

// ----------------------------------------------------- compile-time plans --
// Transform lengths known at compile time get a fully unrolled plan: radix
// sequence, strides, butterflies per thread and twiddle steps are constants,
// which keeps the pass working set in registers.
struct CtPlan {
  int n;
  int np;
  int r[SC_FFT_MAX_PASS];
};

// Radix sequence for compile-time lengths: radix-RM passes (RM = 8 or 16),
// then one smaller power of two, then 3s, 5s, then other primes.
__host__ __device__ constexpr CtPlan ct_plan(int n, int RM) {
  CtPlan p{n, 0, {}};
  int m = n, a = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  const int lr = RM == 16 ? 4 : 3;
  for (int i = 0; i < a / lr; ++i) p.r[p.np++] = RM;
  const int rem = a % lr;
  if (rem > 0) p.r[p.np++] = 1 << rem;
  while (m % 3 == 0) { m /= 3; p.r[p.np++] = 3; }
  while (m % 5 == 0) { m /= 5; p.r[p.np++] = 5; }
  for (int f = 7; m > 1 && p.np < SC_FFT_MAX_PASS; f += 2) {
    while (m % f == 0 && p.np < SC_FFT_MAX_PASS) { m /= f; p.r[p.np++] = f; }
  }
  return p;
}

__host__ __device__ constexpr int ct_ns(const CtPlan& p, int k) {
  int ns = 1;
  for (int i = 0; i < k; ++i) ns *= p.r[i];
  return ns;
}

__host__ __device__ constexpr int ct_pow2ceil(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Threads per transform for a compile-time length: RM elements each (one
// radix-RM butterfly per pass), at least 8 threads.
__host__ __device__ constexpr int ct_threads(int n, int RM) {
  int g = (n + RM - 1) / RM;
  return g < 8 ? 8 : g;
}

// Shared-memory slot of element i of a compile-time transform.
//  * One transform per slot run (ST == 1, the row pass), N a multiple of 16:
//    an XOR swizzle inside every aligned block of 16 elements, slot =
//    i ^ g(i >> 4), with g(x) = (x & 7) | (x & 4) << 1 for radix-8 plans
//    and g(x) = x & 15 for radix-16 plans.  A half-warp of 8-byte accesses
//    is conflict-free when it touches 16 contiguous aligned elements (every
//    load, the stores of the later passes) or the stores of the first pass
//    (elements R j + q of 16 consecutive butterflies j); with radix 8 also
//    two runs of 8 elements 64 apart (stores of the second pass).  No
//    padding.
//  * Interleaved transforms (ST > 1, the column pass, ST columns of 8 bytes
//    per slot): one pad slot after every ct_pad elements (the first radix),
//    which spreads the strided stores of the first pass over all banks.
__host__ __device__ constexpr int ct_pad(int n, int RM) { return ct_plan(n, RM).r[0]; }
__host__ __device__ constexpr bool ct_swizzled(int n, int ST) { return ST == 1 && n % 16 == 0; }
// g of the swizzled layout; linear over GF(2): g(a ^ b) = g(a) ^ g(b).
template <int RM>
__host__ __device__ constexpr int ct_swz(int x) {
  return RM == 16 ? (x & 15) : ((x & 7) | ((x & 4) << 1));
}
// Index period of the swizzle pattern (g reads bits 4..7 or 4..6 of i).
__host__ __device__ constexpr int ct_swz_period(int RM) { return RM == 16 ? 256 : 128; }
template <int N, int RM, int ST>
__device__ __forceinline__ int ct_phys(int i) {
  if constexpr (ct_swizzled(N, ST)) {
    return i ^ ct_swz<RM>(i >> 4);
  } else {
    constexpr int P = ct_pad(N, RM);
    return i + i / P;
  }
}
// Shared-memory slots (elements) of one compile-time transform.
__host__ __device__ constexpr int ct_padded(int n, int RM) { return n + n / ct_pad(n, RM); }
__host__ __device__ constexpr int ct_len(int n, int RM, int ST) {
  return ct_swizzled(n, ST) ? n : ct_padded(n, RM);
}

// Slot of element i0 + q * STRIDE (q < Q, compile-time) from the slot of i0.
// In the swizzled layout:
//  * a stride that is a multiple of the swizzle period keeps the pattern:
//    slot = slot(i0) + q STRIDE;
//  * STRIDE and Q powers of two and i0 sharing no bit with q STRIDE (the
//    callers' butterflies: loads j + q B with j < B, stores base + q NS with
//    base = (j - j % NS) R + j % NS, first-pass stores R t + q): i0 + q
//    STRIDE = i0 | q STRIDE and g is linear, so slot = slot(i0) ^ q STRIDE ^
//    g(q STRIDE >> 4), a compile-time constant per q (an add folded into the
//    address when STRIDE >= 16).
// Otherwise the slot is computed per element.
template <int N, int RM, int ST, int STRIDE, int Q>
struct CtRun {
  static constexpr bool pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }
  static constexpr bool add = ct_swizzled(N, ST) && STRIDE % ct_swz_period(RM) == 0;
  static constexpr bool lin = ct_swizzled(N, ST) && pow2(STRIDE) && pow2(Q);
  __device__ __forceinline__ static int base(int i0) { return ct_phys<N, RM, ST>(i0); }
  __device__ __forceinline__ static int at(int s0, int i0, int q) {
    if constexpr (add) {
      return s0 + q * STRIDE;
    } else if constexpr (lin) {
      if constexpr (STRIDE >= 16) return (s0 ^ ct_swz<RM>((q * STRIDE) >> 4)) + q * STRIDE;
      else return s0 ^ ((q * STRIDE) ^ ct_swz<RM>((q * STRIDE) >> 4));
    } else {
      return ct_phys<N, RM, ST>(i0 + q * STRIDE);
    }
  }
};

template <int N, int RM, int R, int NS, int G, int ST>
__device__ __forceinline__ void ct_pass(float2* data, const float2* __restrict__ tw, int t) {
  constexpr int B = N / R;
  constexpr int NB = (B + G - 1) / G;
  constexpr int STEP = N / (NS * R);
  float2 v[NB][R];
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = t + i * G;
    if ((B % G) == 0 || j < B) {
      using LD = CtRun<N, RM, ST, B, R>;
      const int s0 = LD::base(j);
#pragma unroll
      for (int q = 0; q < R; ++q) v[i][q] = data[LD::at(s0, j, q) * ST];
      if constexpr (NS > 1) twiddle_r<R>(v[i], tw, (j % NS) * STEP);
      dft_r<R>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = t + i * G;
    if ((B % G) == 0 || j < B) {
      const int k = j % NS;
      const int base = (j - k) * R + k;
      using SD = CtRun<N, RM, ST, NS, R>;
      const int s0 = SD::base(base);
#pragma unroll
      for (int q = 0; q < R; ++q) data[SD::at(s0, base, q) * ST] = v[i][q];
    }
  }
  __syncthreads();
}

template <int N, int RM, int G, int ST, int P = 0>
__device__ __forceinline__ void fft_ct(float2* data, const float2* __restrict__ tw, int t) {
  constexpr CtPlan pl = ct_plan(N, RM);
  if constexpr (P < pl.np) {
    ct_pass<N, RM, pl.r[P], ct_ns(pl, P), G, ST>(data, tw, t);
    fft_ct<N, RM, G, ST, P + 1>(data, tw, t);
  }
}

// Passes [P, PEND) of a compile-time plan.
template <int N, int RM, int G, int ST, int P, int PEND>
__device__ __forceinline__ void fft_ct_passes(float2* data, const float2* __restrict__ tw, int t) {
  constexpr CtPlan pl = ct_plan(N, RM);
  if constexpr (P < PEND) {
    ct_pass<N, RM, pl.r[P], ct_ns(pl, P), G, ST>(data, tw, t);
    fft_ct_passes<N, RM, G, ST, P + 1, PEND>(data, tw, t);
  }
}

// A compile-time transform whose first radix is N/G and whose last pass has
// a stride N/R_last that is a multiple of G gives thread t the elements
// t + G m (m < N/G) both as the inputs of its first pass and as the outputs
// of its last pass.  Two transforms in a row can then hand over in
// registers: the last pass of one, an element-wise step and the first pass
// of the next need no shared-memory round trip (powers of two from 64 with
// radix-8 plans).
__host__ __device__ constexpr bool ct_reg_edges(int n, int RM) {
  const CtPlan p = ct_plan(n, RM);
  const int G = ct_threads(n, RM);
  return p.np >= 2 && n % G == 0 && p.r[0] == n / G && (n / p.r[p.np - 1]) % G == 0;
}

// First pass of a compile-time transform with its inputs in registers,
// v[m] = element t + G m; results stored to shared memory.  Starts with a
// barrier, so callers may still be reading the data array.
template <int N, int RM, int ST>
__device__ __forceinline__ void ct_first_from_regs(float2* data, float2* v, int t) {
  constexpr CtPlan pl = ct_plan(N, RM);
  constexpr int R = pl.r[0];
  dft_r<R>(v);  // Ns = 1: no twiddles; butterfly j = t takes t + G q
  __syncthreads();
  const int base = t * R;
  using SD = CtRun<N, RM, ST, 1, R>;
  const int s0 = SD::base(base);
#pragma unroll
  for (int q = 0; q < R; ++q) data[SD::at(s0, base, q) * ST] = v[q];
  __syncthreads();
}

// Last pass of a compile-time transform with its outputs left in registers,
// v[m] = element t + G m.  Reads shared memory only.
template <int N, int RM, int ST>
__device__ __forceinline__ void ct_last_to_regs(const float2* data,
                                                const float2* __restrict__ tw, float2* v,
                                                int t) {
  constexpr CtPlan pl = ct_plan(N, RM);
  constexpr int G = ct_threads(N, RM);
  constexpr int PL = pl.np - 1;
  constexpr int R = pl.r[PL];
  constexpr int NS = ct_ns(pl, PL);  // = N / R: butterfly j's outputs are j + NS q
  constexpr int NB = NS / G;
  constexpr int STEP = N / (NS * R);
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = t + i * G;
    float2 u[R];
    using LD = CtRun<N, RM, ST, NS, R>;
    const int s0 = LD::base(j);
#pragma unroll
    for (int q = 0; q < R; ++q) u[q] = data[LD::at(s0, j, q) * ST];
    twiddle_r<R>(u, tw, (j % NS) * STEP);
    dft_r<R>(u);
#pragma unroll
    for (int q = 0; q < R; ++q) v[i + NB * q] = u[q];
  }
}

// Forward DFT of length N of the elements of one transform (N > 0:
// compile-time plan with radix-RM passes, element i at
// data[ct_phys<N, RM>(i) * ST]; N == 0: runtime plan P with g threads,
// element i at data[i * ST]).
template <int N, int ST, int RM>
__device__ __forceinline__ void fft_any(float2* data, const FftPlan& P,
                                        const float2* __restrict__ tw, int t, int g) {
  if constexpr (N == 0) {
    fft_forward<16>(data, P, ST, tw, t, g);
  } else {
    fft_ct<N, RM, ct_threads(N, RM), ST>(data, tw, t);
  }
}

// Element index -> shared-memory slot for either path (ST: transforms
// interleaved per slot, as passed to fft_any).
template <int N, int RM, int ST>
__device__ __forceinline__ int fft_slot(int i) {
  if constexpr (N == 0) return i;
  else return ct_phys<N, RM, ST>(i);
}
