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
//   8-byte elements (complex float): p ^ ((p >> 4) & 15), a permutation inside each 128-byte line
//   (16 elements) keyed by the line index: the contiguous reads of every stage stay on whole
//   lines (two wavefronts per warp) and the stride-E writes of stage 0 and the grouped writes of
//   the middle stages spread over all 32 banks (two wavefronts for N = 256, E = 8).
//   16-byte elements (complex double): one spare slot per E elements (p + p / E), which spreads
//   the stride-E writes; a warp needs four wavefronts for these anyway.
// Without PAD: p (column buffers, sstride = columns per block).
template <typename T, int E, bool PAD> __device__ __forceinline__ int sidx(int p) {
  if constexpr (!PAD) return p;
  else if constexpr (sizeof(T) == 4) return p ^ ((p >> 4) & 15);
  else return p + (p >> ilog2(E));
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
    for (int r = 0; r < R; ++r) x[q * R + r] = sbuf[sidx<T, E, PAD>(b + r * (N / R)) * sstride];
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
      for (int r = 0; r < R; ++r) sbuf[sidx<T, E, PAD>(base + r * Ns) * sstride] = x[q * R + r];
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
  using Sh = FftShape<N, E>;
  dft<T, E, INV>(a);  // stage 0: radix E, Ns = 1, no twiddles
  if constexpr (Sh::S > 1) {
#pragma unroll
    for (int r = 0; r < E; ++r) sbuf[sidx<T, E, PAD>(j * E + r) * sstride] = a[r];
    sync();
    fft_stage<T, N, E, INV, PAD, 1>(a, sbuf, sstride, j, tw, sync);
  }
}

}  // namespace ld
