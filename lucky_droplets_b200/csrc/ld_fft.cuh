// In-register radix-R DFTs and a Stockham autosort engine for batched length-N complex FFTs.
//
// Thread model: one FFT of length N is computed by NT = N / E cooperating threads, each holding
// E elements.  The first stage is radix E (one butterfly per thread); later stages are radix E
// except a shorter last one (N need not be a power of E).  Between stages the threads exchange
// through a caller-provided shared-memory column (element p at sbuf[p * sstride]).
//
// Register contract of fft_run():
//   on entry  a[m] = x[j + NT*m]      (m = 0..E-1, j = this thread's index within the FFT)
//   on return a[m] = X[j + NT*m]      (same positions, transformed)
// so a thread's outputs sit at exactly the positions of its inputs; a forward transform can be
// chained after an inverse one with no exchange in between.
//
// Twiddles for stages >= 1 come from a table tw[p] = exp(-2 pi i p / N), p < N, computed on the
// host in FP64 (and rounded once to the element type).  The radix-R butterflies use the exact
// constants cos(2 pi m / 16), sin(2 pi m / 16).
//
// Lengths that are not powers of two (N = 2^a 3^b 5^c, E a power of two dividing N) take the
// mixed-radix Stockham pipeline below (fft_run_mr): stage 0 is radix E in registers as above;
// the remaining factor N / E is split into radix 8/4/2 stages, then radix 5, then radix 3 stages,
// each stage's N / R butterflies dealt round-robin to the NT threads (a thread does up to
// ceil(N / R / NT) of them; the rest idle), every stage reading and writing the exchange buffer;
// the last stage writes natural order and each thread reads back its own positions, so the
// register contract is the same.
#pragma once
#include "ld_common.cuh"

namespace ld {

__host__ __device__ constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }
__host__ __device__ constexpr int nstages(int n, int e) { return n <= e ? 1 : 1 + nstages(n / e, e); }

template <int N, int E> struct FftShape {
  static_assert((N & (N - 1)) == 0 && (E & (E - 1)) == 0, "powers of two only");
  static_assert(E >= 2 && E <= 16 && E <= N, "radix 2..16");
  static constexpr int NT = N / E;
  static constexpr int S = nstages(N, E);
  static constexpr int RL = N / ipow(E, S - 1);  // radix of the last stage
  static __host__ __device__ constexpr int radix(int s) { return s < S - 1 ? E : RL; }
  static __host__ __device__ constexpr int ns(int s) { return ipow(E, s); }
};

// W_16^m = exp(-2 pi i m / 16) for m = 0..7 (forward sign).  INV conjugates.
template <typename T, bool INV> __device__ __forceinline__ cplx<T> w16mul(cplx<T> x, int m) {
  constexpr T c1 = T(0.92387953251128675613);  // cos(pi/8)
  constexpr T s1 = T(0.38268343236508977173);  // sin(pi/8)
  constexpr T c2 = T(0.70710678118654752440);  // cos(pi/4)
  const T sg = INV ? T(1) : T(-1);             // sign of the sine part
  switch (m) {
    case 0: return x;
    case 4: return INV ? cmk(-x.y, x.x) : cmk(x.y, -x.x);  // * (+-i)
    case 2: { T a = x.x, b = x.y;                            // * c2 (1 -+ i)
      return INV ? cmk(c2 * (a - b), c2 * (a + b)) : cmk(c2 * (a + b), c2 * (b - a)); }
    case 6: { T a = x.x, b = x.y;                            // * c2 (-1 -+ i)
      return INV ? cmk(-c2 * (a + b), c2 * (a - b)) : cmk(c2 * (b - a), -c2 * (a + b)); }
    default: {
      T wr, wi;
      switch (m) {
        case 1: wr = c1;  wi = s1; break;
        case 3: wr = s1;  wi = c1; break;
        case 5: wr = -s1; wi = c1; break;
        default: wr = -c1; wi = s1; break;  // m == 7
      }
      wi *= sg;
      return cmk(x.x * wr - x.y * wi, x.x * wi + x.y * wr);
    }
  }
}

__host__ __device__ constexpr int bitrev(int i, int bits) {
  return bits == 0 ? 0 : ((i & 1) << (bits - 1)) | bitrev(i >> 1, bits - 1);
}
__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

// One radix-2 pass (butterfly span LEN) of an in-place length-R DIT DFT, then the next pass.
// LEN is a template constant so every loop has a compile-time trip count and every index into
// a[] is static: the array stays in registers.
template <typename T, int R, int LEN, bool INV> __device__ __forceinline__ void dft_pass(cplx<T>* a) {
  if constexpr (LEN <= R) {
#pragma unroll
    for (int i = 0; i < R; i += LEN) {
#pragma unroll
      for (int q = 0; q < LEN / 2; ++q) {
        const cplx<T> u = a[i + q];
        const cplx<T> v = w16mul<T, INV>(a[i + q + LEN / 2], q * (16 / LEN));
        a[i + q] = cadd(u, v);
        a[i + q + LEN / 2] = csub(u, v);
      }
    }
    dft_pass<T, R, 2 * LEN, INV>(a);
  }
}

// Bit-reversal permutation of a[0..R-1], one compile-time swap at a time.
template <typename T, int R, int I> __device__ __forceinline__ void bitrev_swaps(cplx<T>* a) {
  if constexpr (I < R) {
    constexpr int K = bitrev(I, ilog2(R));
    if constexpr (K > I) {
      const cplx<T> t = a[I];
      a[I] = a[K];
      a[K] = t;
    }
    bitrev_swaps<T, R, I + 1>(a);
  }
}

// In-place length-R DFT of a[0..R-1] (natural order in and out), R in {1,2,4,8,16}.
template <typename T, int R, bool INV> __device__ __forceinline__ void dft(cplx<T>* a) {
  if constexpr (R > 1) {
    bitrev_swaps<T, R, 0>(a);
    dft_pass<T, R, 2, INV>(a);
  }
}

// Twiddle exp(-+2 pi i p / N) from the FP64-built table.
template <typename T, bool INV> __device__ __forceinline__ cplx<T> twid(const cplx<T>* tw, int p) {
  cplx<T> w = tw[p];
  if (INV) w.y = -w.y;
  return w;
}

// Barrier kinds for the exchanges.
// Each barrier is bracketed by compiler memory clobbers so that no shared-memory access of the
// exchange is moved across it.
struct SyncBlock {
  __device__ __forceinline__ void operator()() const {
    asm volatile("" ::: "memory");
    __syncthreads();
    asm volatile("" ::: "memory");
  }
};
struct SyncWarp {
  __device__ __forceinline__ void operator()() const {
    asm volatile("" ::: "memory");
    __syncwarp();
    asm volatile("" ::: "memory");
  }
};

// Shared-memory slot of element p of a row buffer (sstride = 1) when PAD is set.
//   8-byte elements (complex float): p ^ mask(p / 16), a permutation inside each 128-byte line
//   (16 elements) keyed by the line index: the contiguous reads of every stage stay on whole
//   lines (two wavefronts per warp) and the stride-E writes of stage 0 and the grouped writes of
//   the middle stages spread over the banks.  A warp's 8-byte accesses are served half a warp at
//   a time, so the sixteen elements of each half must fall in distinct bank pairs: mask = the
//   line index (p >> 4) & 15 achieves it for every access but the stage-1 writes of N = 256,
//   E = 8 (two-way conflicts), which the mixed mask below removes for that size.
//   16-byte elements (complex double): one spare slot per E elements (p + p / E), which spreads
//   the stride-E writes; a warp needs four wavefronts for these anyway.
// Without PAD: p (column buffers, sstride = columns per block).
template <typename T, int N, int E, bool PAD> __device__ __forceinline__ int sidx(int p) {
  if constexpr (!PAD) {
    return p;
  } else if constexpr (sizeof(T) == 4 && N == 256 && E == 8) {
    // 256-point rows of 32 threads (the fused z pass at 256^3): the line index b mixed with b << 1
    // (checked over that row's accesses of 8-byte elements — stage-0 and stage-1 writes, stage-1
    // and stage-2 reads, the forward pair's split — by enumerating each half-warp's bank pairs)
    const int b = (p >> 4) & 15;
    return p ^ ((b ^ (b << 1)) & 15);
  } else if constexpr (sizeof(T) == 4) {
    return p ^ ((p >> 4) & 15);
  } else {
    return p + (p >> ilog2(E));
  }
}

// In-place length-3 and length-5 DFTs (forward sign exp(-2 pi i jk / R); INV conjugates).  The
// constants are cos and sin of 2 pi / 3, 2 pi / 5 and 4 pi / 5.
template <typename T, bool INV> __device__ __forceinline__ void dft3(cplx<T>* x) {
  constexpr T s3 = T(0.86602540378443864676);  // sin(2 pi / 3)
  const cplx<T> t1 = cadd(x[1], x[2]);
  const cplx<T> d = csub(x[1], x[2]);
  const cplx<T> m = cmk(x[0].x - T(0.5) * t1.x, x[0].y - T(0.5) * t1.y);
  // -i s3 d (forward) / +i s3 d (inverse)
  const cplx<T> r = INV ? cmk(-s3 * d.y, s3 * d.x) : cmk(s3 * d.y, -s3 * d.x);
  x[0] = cadd(x[0], t1);
  x[1] = cadd(m, r);
  x[2] = csub(m, r);
}

template <typename T, bool INV> __device__ __forceinline__ void dft5(cplx<T>* x) {
  constexpr T c1 = T(0.30901699437494742410);   // cos(2 pi / 5)
  constexpr T c2 = T(-0.80901699437494742410);  // cos(4 pi / 5)
  constexpr T s1 = T(0.95105651629515357212);   // sin(2 pi / 5)
  constexpr T s2 = T(0.58778525229247312917);   // sin(4 pi / 5)
  const cplx<T> a1 = cadd(x[1], x[4]), a2 = cadd(x[2], x[3]);
  const cplx<T> b1 = csub(x[1], x[4]), b2 = csub(x[2], x[3]);
  const cplx<T> t1 = cmk(x[0].x + c1 * a1.x + c2 * a2.x, x[0].y + c1 * a1.y + c2 * a2.y);
  const cplx<T> t2 = cmk(x[0].x + c2 * a1.x + c1 * a2.x, x[0].y + c2 * a1.y + c1 * a2.y);
  const cplx<T> u1 = cmk(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
  const cplx<T> u2 = cmk(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
  // forward: X1 = t1 - i u1, X4 = t1 + i u1, X2 = t2 - i u2, X3 = t2 + i u2
  const cplx<T> iu1 = INV ? cmk(-u1.y, u1.x) : cmk(u1.y, -u1.x);
  const cplx<T> iu2 = INV ? cmk(-u2.y, u2.x) : cmk(u2.y, -u2.x);
  x[0] = cadd(x[0], cadd(a1, a2));
  x[1] = cadd(t1, iu1);
  x[4] = csub(t1, iu1);
  x[2] = cadd(t2, iu2);
  x[3] = csub(t2, iu2);
}

// Any radix of the mixed-radix pipeline: 2, 4, 8, 16 (bit-reversed passes), 3 or 5.
template <typename T, int R, bool INV> __device__ __forceinline__ void dft_any(cplx<T>* x) {
  if constexpr (R == 3) dft3<T, INV>(x);
  else if constexpr (R == 5) dft5<T, INV>(x);
  else dft<T, R, INV>(x);
}

__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
// radix of the next stage for a remaining factor m: 8, 4, 2 first, then 5, then 3
__host__ __device__ constexpr int mr_pick(int m) {
  return m % 8 == 0 ? 8 : (m % 4 == 0 ? 4 : (m % 2 == 0 ? 2 : (m % 5 == 0 ? 5 : (m % 3 == 0 ? 3 : m))));
}
// remaining factor before stage s (s >= 1) of a length-N pipeline whose stage 0 is radix E
__host__ __device__ constexpr int mr_rest(int N, int E, int s) {
  return s <= 1 ? N / E : mr_rest(N, E, s - 1) / mr_pick(mr_rest(N, E, s - 1));
}
__host__ __device__ constexpr int mr_nstages(int m) { return m <= 1 ? 0 : 1 + mr_nstages(m / mr_pick(m)); }
// m is a product of 2s, 3s and 5s
__host__ __device__ constexpr bool mr_ok(int m) {
  return m == 1 || (m > 1 && ((m % 2 == 0 && mr_ok(m / 2)) || (m % 3 == 0 && mr_ok(m / 3)) || (m % 5 == 0 && mr_ok(m / 5))));
}

template <int N, int E> struct MrShape {
  static_assert(is_pow2(E) && E >= 2 && E <= 16 && N % E == 0, "stage 0: a power-of-two radix dividing N");
  static_assert(mr_ok(N / E), "N / E must factor into 2, 3 and 5");
  static constexpr int NT = N / E;
  static constexpr int S = 1 + mr_nstages(N / E);
  static __host__ __device__ constexpr int radix(int s) { return s == 0 ? E : mr_pick(mr_rest(N, E, s)); }
  static __host__ __device__ constexpr int ns(int s) { return N / mr_rest(N, E, s); }  // product of earlier radices
};

// Stage s >= 1 of the mixed-radix pipeline.
template <typename T, int N, int E, bool INV, bool PAD, int s, class Sync>
__device__ __forceinline__ void fft_stage_mr(cplx<T>* a, cplx<T>* sbuf, int sstride, int j,
                                             const cplx<T>* __restrict__ tw, Sync sync) {
  using Sh = MrShape<N, E>;
  constexpr int NT = Sh::NT;
  constexpr int R = Sh::radix(s);
  constexpr int Ns = Sh::ns(s);
  constexpr int NB = N / R;                  // butterflies of this stage
  constexpr int Q = (NB + NT - 1) / NT;      // butterflies per thread
  constexpr bool FULL = Q * NT == NB;
  constexpr bool LAST = s == Sh::S - 1;
  cplx<T> x[Q * R];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = j + NT * q;
    if (FULL || b < NB) {
#pragma unroll
      for (int r = 0; r < R; ++r) x[q * R + r] = sbuf[sidx<T, N, E, PAD>(b + r * NB) * sstride];
    }
  }
  sync();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = j + NT * q;
    if (FULL || b < NB) {
      const int k = b % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) x[q * R + r] = cmul(x[q * R + r], twid<T, INV>(tw, r * k * (N / (Ns * R))));
      dft_any<T, R, INV>(x + q * R);
      // Stockham output position (b / Ns) Ns R + k + r Ns; in the last stage b < Ns, which is
      // natural order b + r NB
      const int base = LAST ? b : (b / Ns) * Ns * R + k;
      constexpr int step = LAST ? NB : Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) sbuf[sidx<T, N, E, PAD>(base + r * step) * sstride] = x[q * R + r];
    }
  }
  sync();
  if constexpr (!LAST) {
    fft_stage_mr<T, N, E, INV, PAD, s + 1>(a, sbuf, sstride, j, tw, sync);
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) a[m] = sbuf[sidx<T, N, E, PAD>(j + NT * m) * sstride];
  }
}

// Stage s >= 1 of the Stockham pipeline (compile-time recursion over the stages).
template <typename T, int N, int E, bool INV, bool PAD, int s, class Sync>
__device__ __forceinline__ void fft_stage(cplx<T>* a, cplx<T>* sbuf, int sstride, int j,
                                          const cplx<T>* __restrict__ tw, Sync sync) {
  using Sh = FftShape<N, E>;
  constexpr int NT = Sh::NT;
  constexpr int S = Sh::S;
  constexpr int R = Sh::radix(s);
  constexpr int Ns = Sh::ns(s);
  constexpr int Q = E / R;
  cplx<T> x[E];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = j + NT * q;
#pragma unroll
    for (int r = 0; r < R; ++r) x[q * R + r] = sbuf[sidx<T, N, E, PAD>(b + r * (N / R)) * sstride];
  }
  sync();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = j + NT * q;
    const int k = b % Ns;
#pragma unroll
    for (int r = 1; r < R; ++r) x[q * R + r] = cmul(x[q * R + r], twid<T, INV>(tw, r * k * (N / (Ns * R))));
    dft<T, R, INV>(x + q * R);
    if constexpr (s < S - 1) {
      const int base = (b / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) sbuf[sidx<T, N, E, PAD>(base + r * Ns) * sstride] = x[q * R + r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) a[q + r * Q] = x[q * R + r];
    }
  }
  if constexpr (s < S - 1) {
    sync();
    fft_stage<T, N, E, INV, PAD, s + 1>(a, sbuf, sstride, j, tw, sync);
  }
}

// Full FFT of length N; see the register contract at the top of this file.  The caller must
// not touch sbuf between fft_run() calls without a barrier: the last stage reads it.
template <typename T, int N, int E, bool INV, bool PAD, class Sync>
__device__ __forceinline__ void fft_run(cplx<T>* a, cplx<T>* sbuf, int sstride, int j,
                                        const cplx<T>* __restrict__ tw, Sync sync) {
  dft<T, E, INV>(a);  // stage 0: radix E, Ns = 1, no twiddles
  if constexpr (is_pow2(N)) {
    using Sh = FftShape<N, E>;
    if constexpr (Sh::S > 1) {
#pragma unroll
      for (int r = 0; r < E; ++r) sbuf[sidx<T, N, E, PAD>(j * E + r) * sstride] = a[r];
      sync();
      fft_stage<T, N, E, INV, PAD, 1>(a, sbuf, sstride, j, tw, sync);
    }
  } else {
    static_assert(MrShape<N, E>::S > 1, "mixed-radix lengths have later stages");
#pragma unroll
    for (int r = 0; r < E; ++r) sbuf[sidx<T, N, E, PAD>(j * E + r) * sstride] = a[r];
    sync();
    fft_stage_mr<T, N, E, INV, PAD, 1>(a, sbuf, sstride, j, tw, sync);
  }
}

}  // namespace ld
