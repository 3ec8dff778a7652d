// Kernel templates of the DNS step: the three axis passes of the 3D real transform, the fused
// nonlinear-term z pass, the k-space update epilogues, spectra/forcing and the droplet kernels.
//
// Data layout (see include/ld.h): physical fields (N,N,N) z fastest; spectra either in the
// reference's full layout (N, N, Nf) or in the dealiased cube (Mx, My, Mzp).
//
// Transform structure for the DNS (cube layout, c = complex element):
//   inverse : x pass (cube rows kx -> N rows x)  |  y pass (My rows ky -> N rows y)
//             |  z pass (kz <= kc -> N reals z)
//   forward : z pass (N reals -> kz < Mzp)  |  y pass (N rows -> My rows)  |  x pass (N -> Mx)
// Rows that are zero on input (|k| > kc) are never read and rows outside the cube are never
// written, so each pass moves only the data the dealiased spectrum needs.
#pragma once
#include <type_traits>

#include "ld_async.cuh"
#include "ld_fft.cuh"

namespace ld {

// ------------------------------------------------------------------------------------------
// index helpers
// ------------------------------------------------------------------------------------------
// logical FFT index n in [0, N) -> compact cube row, or -1 when |freq| > kc
__device__ __forceinline__ int crow(int n, int N, int kc) {
  return n <= kc ? n : (n >= N - kc ? n - (N - 2 * kc - 1) : -1);
}
// compact cube row -> signed frequency
__device__ __forceinline__ int cfreq(int i, int kc) { return i <= kc ? i : i - (2 * kc + 1); }
// logical FFT index -> signed frequency (fftfreq convention: N/2 -> -N/2)
__device__ __forceinline__ int nfreq(int n, int N) { return n < N / 2 ? n : n - N; }

// 4-vectors for interleaved physical fields (u, v, w, 0)
template <typename T> struct V4T;
template <> struct V4T<float> { using type = float4; };
template <> struct V4T<double> { using type = double4; };
template <typename T> using vec4 = typename V4T<T>::type;
template <typename T> __device__ __forceinline__ vec4<T> mk4(T a, T b, T c, T d) {
  vec4<T> v; v.x = a; v.y = b; v.z = c; v.w = d; return v;
}

// Launch shapes by N.  Powers of two: as tuned.  Mixed-radix N = 2^a 3^b 5^c (a >= 3): eight
// elements per thread (stage 0 radix 8) in both kinds of pass; column passes with a CTA of 8
// columns (64-byte FP32 / 128-byte FP64 row segments; N/8 x 8 threads leave the FP64 update pass,
// which holds three transformed columns, enough registers); z passes with as many row units per
// CTA as fit 256 threads (a power of two, so that N^2 rows split evenly); their rows span warps,
// so they exchange with block-wide barriers.  (Measured at 360^3 in FP64 against four elements
// per thread, two or three CTAs per SM and a block-pipelined variant with bulk-copy prefetch:
// this shape was the fastest of them.)
template <int N> struct Cfg {
  static constexpr bool P2 = is_pow2(N);
  // column passes: E elements per thread, TB columns per CTA
  static constexpr int EC = P2 ? ((N == 32 || N == 64) ? 8 : 16) : 8;
  static constexpr int NTC = N / EC;
  static constexpr int TB = P2 ? (N == 16 ? 64 : (N == 32 ? 32 : 16)) : 8;
  static constexpr int COL_THREADS = TB * NTC;
  // z passes: E elements per thread, NTZ threads per row
  static constexpr int EZ = P2 ? (N >= 512 ? 16 : 8) : 8;
  static constexpr int NTZ = N / EZ;
  static constexpr int ZROWS = P2 ? 256 / NTZ : (256 / NTZ >= 16 ? 16 : (256 / NTZ >= 8 ? 8 : (256 / NTZ >= 4 ? 4 : (256 / NTZ >= 2 ? 2 : 1))));
  static constexpr int ZTHREADS = ZROWS * NTZ;  // row units per CTA x threads per row
  static constexpr int LOGEZ = ilog2(EZ);
  // the dealiased cube of a plan of size N (ld_plan_create: kc = N / 3, rows padded to 8)
  static constexpr int KC = N / 3;
  static constexpr int MY = 2 * KC + 1;
  static constexpr int MZP = (KC + 1 + 7) / 8 * 8;
  static constexpr int ZBUF = N + N / EZ;       // padded row buffer (bank-conflict free)
};

// ------------------------------------------------------------------------------------------
// column (strided axis) passes
// ------------------------------------------------------------------------------------------
// Plain strided loader/storer: element (f, o, row, col) at f*fs + o*os + row*rs + col, with an
// optional cube row map (kc >= 0) on the transform axis.
template <typename T> struct RowsIO {
  cplx<T>* p;
  long long fs, os;
  int rs;
  int kc;  // < 0: identity row map
  __device__ __forceinline__ long long at(int f, int o, int r, int col) const {
    return (long long)f * fs + (long long)o * os + (long long)r * rs + col;
  }
};


// Strided row loader and storer with the row map chosen at run time (io.kc < 0: rows as they are,
// else compact cube rows through crow).
template <typename T, int N> struct LdRows {
  RowsIO<T> io;
  __device__ __forceinline__ cplx<T> operator()(int f, int o, int n, int col) const {
    const int r = io.kc < 0 ? n : crow(n, N, io.kc);
    if (r < 0) return czero<cplx<T>>();
    return io.p[io.at(f, o, r, col)];
  }
};

template <typename T, int N> struct StRows {
  RowsIO<T> io;
  __device__ __forceinline__ void operator()(int f, int o, int n, int col, cplx<T> v) const {
    const int r = io.kc < 0 ? n : crow(n, N, io.kc);
    if (r < 0) return;
    io.p[io.at(f, o, r, col)] = v;
  }
};

// Strided row loader: rows mapped to compact cube rows through crow (MAP) or taken as they are.
template <typename T, int N, bool MAP> struct LdRowsC {
  RowsIO<T> io;
  __device__ __forceinline__ cplx<T> operator()(int f, int o, int n, int col) const {
    const int r = MAP ? crow(n, N, Cfg<N>::KC) : n;  // io.kc == Cfg<N>::KC for cube rows
    if (r < 0) return czero<cplx<T>>();
    return io.p[io.at(f, o, r, col)];
  }
};


// Strided row storer: rows mapped to compact cube rows through crow (MAP; rows outside the cube
// are not written) or taken as they are.
template <typename T, int N, bool MAP> struct StRowsC {
  RowsIO<T> io;
  __device__ __forceinline__ void operator()(int f, int o, int n, int col, cplx<T> v) const {
    const int r = MAP ? crow(n, N, Cfg<N>::KC) : n;  // io.kc == Cfg<N>::KC for cube rows
    if (r < 0) return;
    io.p[io.at(f, o, r, col)] = v;
  }
};

// Storer into the cube that also applies the spherical mask round(|k|) <= kc (F:129): the last
// (x) pass of a forward cube transform.  Columns are the flat (ky, kz) index of a kx plane.
template <typename T, int N> struct StCube {
  RowsIO<T> io;  // io.kc = kc (compact rows), io.rs = My * Mzp
  int Mzp;
  __device__ __forceinline__ void operator()(int f, int o, int n, int col, cplx<T> v) const {
    const int kc = io.kc;
    const int r = crow(n, N, kc);
    if (r < 0) return;
    const int kx = n <= kc ? n : n - N;
    const int iy = col / Mzp;
    const int ky = cfreq(iy, kc), kz = col - iy * Mzp;
    if (kz > kc || kx * kx + ky * ky + kz * kz > kc * kc + kc) v = czero<cplx<T>>();
    io.p[io.at(f, o, r, col)] = v;
  }
};

// Inverse x-pass loader producing [u_x, u_y, u_z, w_x, w_y, w_z] from a cube 3-vector:
// w = i k x u (F:295-297).  Columns are the flat (ky, kz) index of a kx plane.
template <typename T, int N> struct LdCurl {
  const cplx<T>* u;
  long long cs;  // component stride (cube elements)
  int kc_, My_, Mzp_;  // the plan's cube; equal to Cfg<N>::KC, MY, MZP, which the loader uses
  long long bs;  // box stride (elements): the outer index is the box of a multi-box plan
  static constexpr int kc = Cfg<N>::KC, My = Cfg<N>::MY, Mzp = Cfg<N>::MZP;
  __device__ __forceinline__ cplx<T> operator()(int f, int o, int n, int col) const {
    const int r = crow(n, N, kc);
    if (r < 0) return czero<cplx<T>>();
    const long long b = (long long)o * bs + (long long)r * My * Mzp + col;
    if (f < 3) return u[f * cs + b];
    const T kx = T(n <= kc ? n : n - N);
    const int iy = col / Mzp;
    const T ky = T(cfreq(iy, kc));
    const T kz = T(col - iy * Mzp);
    cplx<T> w;
    if (f == 3) {        // i (ky u_z - kz u_y)
      cplx<T> uy = u[cs + b], uz = u[2 * cs + b];
      w = cmuli(csub(cscale(uz, ky), cscale(uy, kz)));
    } else if (f == 4) { // i (kz u_x - kx u_z)
      cplx<T> ux = u[b], uz = u[2 * cs + b];
      w = cmuli(csub(cscale(ux, kz), cscale(uz, kx)));
    } else {             // i (kx u_y - ky u_x)
      cplx<T> ux = u[b], uy = u[cs + b];
      w = cmuli(csub(cscale(uy, kx), cscale(ux, ky)));
    }
    return w;
  }
};

// One CTA = TB columns x NT threads; blockIdx.x = tile * nf + field (fields of a tile launch
// together so their shared inputs are served from L2), blockIdx.y = outer index.
template <typename T, int N, bool INV, class Ld, class St>
__global__ void __launch_bounds__(Cfg<N>::COL_THREADS)
k_colfft(Ld ld, St st, int ncols, int nf, const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EC, TB = Cfg<N>::TB, NT = Cfg<N>::NTC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw);
  const int c = threadIdx.x % TB, j = threadIdx.x / TB;
  const int field = blockIdx.x % nf;
  const int col = (blockIdx.x / nf) * TB + c;
  const bool ok = col < ncols;
  const int outer = blockIdx.y;
  cplx<T> a[E];
#pragma unroll
  for (int m = 0; m < E; ++m) a[m] = ok ? ld(field, outer, j + NT * m, col) : czero<cplx<T>>();
  fft_run<T, N, E, INV, false>(a, sbuf + c, TB, j, tw, SyncBlock());
  if (ok) {
#pragma unroll
    for (int m = 0; m < E; ++m) st(field, outer, j + NT * m, col, a[m]);
  }
}

// The same tile (the same body, written out so that k_colfft keeps its code) with five CTAs per
// SM, for N = 256 in FP32: 48 registers, no spills, 32 KB of shared memory each, instead of four
// CTAs at 56 registers.  These one-shot tiles wait on their loads (the inverse x pass with the
// curl stalls mostly on long scoreboard) and the extra warps hide that latency (x inverse
// 0.072 -> 0.067 ms).  Elsewhere k_colfft keeps the compiler's own register choice: stating one
// CTA per SM would let the FP64 tiles grow from about 90 to about 150 registers.
template <typename T, int N, bool INV, class Ld, class St>
__global__ void __launch_bounds__(Cfg<N>::COL_THREADS, 5)
k_colfft5(Ld ld, St st, int ncols, int nf, const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EC, TB = Cfg<N>::TB, NT = Cfg<N>::NTC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw);
  const int c = threadIdx.x % TB, j = threadIdx.x / TB;
  const int field = blockIdx.x % nf;
  const int col = (blockIdx.x / nf) * TB + c;
  const bool ok = col < ncols;
  const int outer = blockIdx.y;
  cplx<T> a[E];
#pragma unroll
  for (int m = 0; m < E; ++m) a[m] = ok ? ld(field, outer, j + NT * m, col) : czero<cplx<T>>();
  fft_run<T, N, E, INV, false>(a, sbuf + c, TB, j, tw, SyncBlock());
  if (ok) {
#pragma unroll
    for (int m = 0; m < E; ++m) st(field, outer, j + NT * m, col, a[m]);
  }
}

template <typename T, int N, bool INV, class Ld, class St>
constexpr auto colfft_kernel() {
  if constexpr (N == 256 && sizeof(T) == 4) return k_colfft5<T, N, INV, Ld, St>;
  else return k_colfft<T, N, INV, Ld, St>;
}

// Pipelined column pass over plain strided rows: a CTA loops over items (column block, field,
// outer index), items of neighbouring CTAs adjacent in memory.  While an item is transformed, the
// rows of the CTA's next item stream into the other shared buffer with 16-byte cp.async copies;
// the buffer an item was staged in serves as its FFT exchange buffer once its values sit in
// registers.  Rows the loader's row map drops (r < 0) and columns past ncols are not copied.
template <typename T, int N, bool INV, class St, bool IN_MAP>
__global__ void __launch_bounds__(Cfg<N>::COL_THREADS, 3)
k_colfft_pipe(RowsIO<T> in, St st, int ncols, int nf, int nouter, const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EC, TB = Cfg<N>::TB, NT = Cfg<N>::NTC;
  constexpr int CPR = TB * (int)sizeof(cplx<T>) / 16;  // 16-byte chunks of a full row segment
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* buf0 = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* buf1 = buf0 + N * TB;
  const int c = threadIdx.x % TB, j = threadIdx.x / TB;
  // item = (column block cb, field f, outer o), cb fastest; the launcher keeps the item count
  // below 2^31, so items are split with 32-bit unsigned division
  const unsigned ncb = (unsigned)((ncols + TB - 1) / TB);
  const unsigned nitems = ncb * (unsigned)nf * (unsigned)nouter;
  struct Item {
    int cb, f, o;
  };
  auto split = [&](unsigned it) {
    const unsigned rest = it / ncb;
    const unsigned fo = rest / (unsigned)nf;
    return Item{(int)(it - rest * ncb), (int)(rest - fo * (unsigned)nf), (int)fo};
  };
  // each thread copies one fixed 16-byte chunk k of rows threadIdx / CPR + (THREADS / CPR) i
  constexpr int THREADS = Cfg<N>::COL_THREADS;
  static_assert(THREADS % CPR == 0 && (N * CPR) % THREADS == 0, "whole rows per pass of the block");
  const int kq = threadIdx.x % CPR, n0 = threadIdx.x / CPR;
  auto prefetch = [&](const Item& itm, cplx<T>* dst) {
    const int col0 = itm.cb * TB;
    const int w = ncols - col0 < TB ? ncols - col0 : TB;
    const int cpr = w * (int)sizeof(cplx<T>) / 16;
    if (kq < cpr) {
      const char* src0 = reinterpret_cast<const char*>(in.p + in.at(itm.f, itm.o, 0, col0)) + 16 * kq;
      const unsigned d0 = (unsigned)__cvta_generic_to_shared(reinterpret_cast<char*>(dst) + 16 * kq);
#pragma unroll
      for (int i = 0; i < N * CPR / THREADS; ++i) {
        const int n = n0 + (THREADS / CPR) * i;
        const int r = IN_MAP ? crow(n, N, in.kc) : n;
        if (r < 0) continue;
        const char* src = src0 + (long long)r * in.rs * (long long)sizeof(cplx<T>);
        const unsigned d = d0 + (unsigned)(n * TB * (int)sizeof(cplx<T>));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  unsigned it = blockIdx.x;
  Item cur_item = split(it);
  if (it < nitems) prefetch(cur_item, buf0);
  int b = 0;
  for (; it < nitems; it += gridDim.x) {
    cplx<T>* cur = b ? buf1 : buf0;
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int f = cur_item.f, o = cur_item.o;
    const int col = cur_item.cb * TB + c;
    const bool ok = col < ncols;
    cplx<T> a[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int n = j + NT * m;
      const int r = IN_MAP ? crow(n, N, in.kc) : n;
      a[m] = (ok && r >= 0) ? cur[n * TB + c] : czero<cplx<T>>();
    }
    __syncthreads();  // every value is in registers: cur becomes the exchange buffer
    const unsigned nx = it + gridDim.x;
    const Item next_item = split(nx);
    if (nx < nitems) prefetch(next_item, b ? buf0 : buf1);
    fft_run<T, N, E, INV, false>(a, cur + c, TB, j, tw, SyncBlock());
    if (ok) {
#pragma unroll
      for (int m = 0; m < E; ++m) st(f, o, j + NT * m, col, a[m]);
    }
    __syncthreads();
    b ^= 1;
    cur_item = next_item;
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------------------------------------------
// k-space update epilogue of the forward x pass (F:304-316 + the time integrators)
// ------------------------------------------------------------------------------------------
enum UpdMode : int {
  UPD_RHS = 0,     // s0 <- P[nl + f] - visc nu k^2 s1               (s1 = stage input)
  UPD_RK2_1 = 1,   // s1 = uk: s0 <- E (uk + h N1) [ustar], s2 <- E (uk + h/2 N1) [acc]
  UPD_RK2_2 = 2,   // s1 = ustar: s0 <- s2 + h/2 N2                   (s0 = uk, s2 = acc)
  UPD_RK4_1 = 3,   // s0 = un, s1 = stage input, s2 = acc, s3 = next stage input
  UPD_RK4_2 = 4,
  UPD_RK4_3 = 5,
  UPD_RK4_4 = 6,
};

template <typename T> struct UpdArgs {
  const cplx<T>* nl;  // forward-transformed (u x w): (3, N, My, Mzp) rows x = N
  long long nls;      // component stride of nl
  cplx<T>* s0;
  cplx<T>* s1;
  cplx<T>* s2;
  cplx<T>* s3;
  long long cs;       // component stride of the cube
  const double* factor;  // forcing factor per shell (FP64), shells kf_lo..kf_hi
  int kf_lo, kf_hi;
  const T* ifac;         // exp(-nu h k^2) by k^2
  T h, nu, visc;
  int kc, My, Mzp;
  unsigned* status;
  // optional slow-manifold velocity of the stage input y (F:319-321):
  // vk = y + tps (k (k . rhs) / k^2 + visc nu k^2 y), minus vg = tps g N^3 on the mean of w
  cplx<T>* vk;
  T tps, vg;
  // RK2 stages: stage the cube rows of the CTA's columns that the update reads (s1 in stage 1,
  // s2 in stage 2) into shared memory with cp.async while the x transforms run; the launcher
  // sets it when the (3, Mx, TB) buffer fits beside the exchange buffer at 2 CTAs per SM
  int prefetch;
  // final stages (UPD_RK2_2, UPD_RK4_4): the step epilogue's work on the kz > 0 modes (projection
  // and the non-finite / blow-up checks, as k_epilogue does them) is done here, so that the
  // epilogue that follows needs only the kz = 0 plane (k_epilogue_plane0)
  T blowup;
  // multi-box plans: blockIdx.y is the box; strides of nl, of the cube states and of the forcing
  // factors from one box to the next
  long long nl_bs, cube_bs;
  int fac_bs;
};

// The step epilogue of one kz > 0 mode (k_epilogue's arithmetic): projection with its own k
// inside the mask, zero outside; flags for non-finite values and the blow-up threshold.
template <typename T>
__device__ __forceinline__ void epi_mode(cplx<T> (&v)[3], int kx, int ky, int kz, int kc, T blowup, unsigned& flags) {
  const int k2 = kx * kx + ky * ky + kz * kz;
  if (kz <= kc && k2 <= kc * kc + kc) {
    const T qx = T(kx), qy = T(ky), qz = T(kz);
    cplx<T> kd = cscale(cadd(cadd(cscale(v[0], qx), cscale(v[1], qy)), cscale(v[2], qz)), T(1) / T(k2));
    v[0] = csub(v[0], cscale(kd, qx));
    v[1] = csub(v[1], cscale(kd, qy));
    v[2] = csub(v[2], cscale(kd, qz));
  } else {
    v[0] = v[1] = v[2] = czero<cplx<T>>();
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!(isfinite(v[c].x) && isfinite(v[c].y))) flags |= LD_STATUS_NONFINITE;
    if (v[c].x > blowup) flags |= LD_STATUS_BLOWUP;
  }
}

template <typename T, int N, int MODE>
__global__ void __launch_bounds__(Cfg<N>::COL_THREADS, (N == 256 && sizeof(T) == 4) ? 2 : 1)
k_xfwd_update(UpdArgs<T> A, int ncols, const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EC, TB = Cfg<N>::TB, NT = Cfg<N>::NTC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (blockIdx.y) {  // box of a multi-box plan
    const long long bo = blockIdx.y;
    A.nl += bo * A.nl_bs;
    if (A.s0) A.s0 += bo * A.cube_bs;
    if (A.s1) A.s1 += bo * A.cube_bs;
    if (A.s2) A.s2 += bo * A.cube_bs;
    if (A.s3) A.s3 += bo * A.cube_bs;
    A.factor += bo * A.fac_bs;
  }
  cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw);
  const int c = threadIdx.x % TB, j = threadIdx.x / TB;
  const int col = blockIdx.x * TB + c;
  const bool ok = col < ncols;
  constexpr bool RK2 = MODE == UPD_RK2_1 || MODE == UPD_RK2_2;
  constexpr int Mx = Cfg<N>::MY;  // A.kc == Cfg<N>::KC, A.My == Cfg<N>::MY, A.Mzp == Cfg<N>::MZP
  cplx<T>* ybuf = sbuf + N * TB;  // (3, Mx, TB) staged rows of s1 (stage 1) or s2 (stage 2)
  const bool pre = RK2 && A.prefetch;
  if (pre) {
    constexpr int PER = 16 / (int)sizeof(cplx<T>);  // elements per 16-byte chunk
    const cplx<T>* src = MODE == UPD_RK2_1 ? A.s1 : A.s2;
    const int col0 = blockIdx.x * TB;
    const int w = ncols - col0 < TB ? ncols - col0 : TB;  // a multiple of 8 (Mzp is)
    const int cpr = w / PER;
    constexpr long long rs = (long long)Cfg<N>::MY * Cfg<N>::MZP;
    for (int q = threadIdx.x; q < 3 * Mx * (TB / PER); q += blockDim.x) {
      const int row = q / (TB / PER), k = q - row * (TB / PER);  // row = cc * Mx + r
      if (k >= cpr) continue;
      const int cc = row / Mx, r = row - cc * Mx;
      const cplx<T>* g = src + cc * A.cs + r * rs + col0 + k * PER;
      const unsigned d = (unsigned)__cvta_generic_to_shared(ybuf + row * TB + k * PER);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  // the three components' loads in flight together, then their transforms (the registers of all
  // three are live through the last transform either way)
  cplx<T> res[3][E];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int m = 0; m < E; ++m)
      res[f][m] = ok ? A.nl[f * A.nls + (long long)(j + NT * m) * ncols + col] : czero<cplx<T>>();
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    if (f) __syncthreads();
    fft_run<T, N, E, false, false>(res[f], sbuf + c, TB, j, tw, SyncBlock());
  }
  if (pre) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
  if (!ok) return;
  const int iy = col / Cfg<N>::MZP;
  const int kzi = col - iy * Cfg<N>::MZP;
  const int kyi = cfreq(iy, Cfg<N>::KC);
  const T ky = T(kyi), kz = T(kzi);
  constexpr int kc = Cfg<N>::KC;
  unsigned flags = 0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = j + NT * m;
    const int r = crow(n, N, kc);
    if (r < 0) continue;
    const int kxi = n <= kc ? n : n - N;
    const T kx = T(kxi);
    const int k2 = kxi * kxi + kyi * kyi + kzi * kzi;
    const long long idx = (long long)r * (Cfg<N>::MY * Cfg<N>::MZP) + col;
    const bool keep = (kzi <= kc) && (k2 <= kc * kc + kc);  // round(|k|) <= kc  (F:129)
    // forcing on shells kf_lo..kf_hi: factor[kint] * y  (F:253-264)
    T fac = T(0);
    if (keep && k2 <= A.kf_hi * A.kf_hi + A.kf_hi) {
      int s = 0;
      while (s * s + s < k2) ++s;  // s = round(sqrt(k2))
      if (s >= A.kf_lo) fac = T(A.factor[s]);
    }
    // the stage input; the second RK2 stage reads it only for the forcing and the slow manifold
    const bool need_y = MODE != UPD_RK2_2 || A.vk != nullptr || fac != T(0);
    cplx<T> y[3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
      y[cc] = !need_y ? czero<cplx<T>>()
                      : ((MODE == UPD_RK2_1 && pre) ? ybuf[(cc * Mx + r) * TB + c] : A.s1[cc * A.cs + idx]);
    cplx<T> rhs[3];
    cplx<T> kd = czero<cplx<T>>();  // (k . rhs) / k^2 before the projection
    if (keep) {
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) rhs[cc] = cadd(res[cc][m], cscale(y[cc], fac));
      if (k2 > 0) {  // pressure projection, invlap = -1/k^2 (F:309-316)
        const T inv = T(1) / T(k2);
        kd = cadd(cadd(cscale(rhs[0], kx), cscale(rhs[1], ky)), cscale(rhs[2], kz));
        kd = cscale(kd, inv);
        rhs[0] = csub(rhs[0], cscale(kd, kx));
        rhs[1] = csub(rhs[1], cscale(kd, ky));
        rhs[2] = csub(rhs[2], cscale(kd, kz));
      }
    } else {
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) rhs[cc] = czero<cplx<T>>();
    }
    if (A.vk) {
      // -i k pk = -k (k . rhs) / k^2 and -nu k^2 y: the reference's Du/Dt of the slow manifold
      const T lvs = A.visc * A.nu * T(k2);
      const T kk[3] = {kx, ky, kz};
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        cplx<T> v = czero<cplx<T>>();
        if (keep) v = cadd(y[cc], cscale(cadd(cscale(kd, kk[cc]), cscale(y[cc], lvs)), A.tps));
        if (cc == 2 && k2 == 0) v.x -= A.vg;
        A.vk[cc * A.cs + idx] = v;
      }
    }
    const T h = A.h;
    if (MODE == UPD_RHS) {
      const T lv = A.visc * A.nu * T(k2);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) A.s0[cc * A.cs + idx] = csub(rhs[cc], cscale(y[cc], lv));
    } else if (MODE == UPD_RK2_1) {
      const T Ef = keep ? A.ifac[k2] : T(0);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        cplx<T> us = cscale(cadd(y[cc], cscale(rhs[cc], h)), Ef);
        cplx<T> ac = cscale(cadd(y[cc], cscale(rhs[cc], T(0.5) * h)), Ef);
        A.s0[cc * A.cs + idx] = us;
        A.s2[cc * A.cs + idx] = ac;
      }
    } else if (MODE == UPD_RK2_2) {
      cplx<T> v[3];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const cplx<T> acc = pre ? ybuf[(cc * Mx + r) * TB + c] : A.s2[cc * A.cs + idx];
        v[cc] = cadd(acc, cscale(rhs[cc], T(0.5) * h));
        if (!keep) v[cc] = czero<cplx<T>>();
        if (!(isfinite(v[cc].x) && isfinite(v[cc].y))) flags |= LD_STATUS_NONFINITE;
      }
      if (kzi > 0) epi_mode(v, kxi, kyi, kzi, kc, A.blowup, flags);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) A.s0[cc * A.cs + idx] = v[cc];
    } else {
      // RK4 (F:341-360): ku = rhs - nu k^2 y ;  y = stage input
      const T lv = A.nu * T(k2);
      cplx<T> ku[3];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) ku[cc] = csub(rhs[cc], cscale(y[cc], lv));
      if (MODE == UPD_RK4_4) {
        cplx<T> v[3];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          v[cc] = cadd(A.s2[cc * A.cs + idx], cscale(ku[cc], h / T(6)));
          if (!(isfinite(v[cc].x) && isfinite(v[cc].y))) flags |= LD_STATUS_NONFINITE;
        }
        if (kzi > 0) epi_mode(v, kxi, kyi, kzi, kc, A.blowup, flags);
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) A.s0[cc * A.cs + idx] = v[cc];
      } else {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const long long o = cc * A.cs + idx;
          if (MODE == UPD_RK4_1) {
            cplx<T> un = y[cc];
            A.s2[o] = cadd(un, cscale(ku[cc], h / T(6)));
            A.s3[o] = cadd(un, cscale(ku[cc], h / T(2)));
          } else {  // UPD_RK4_2, UPD_RK4_3
            cplx<T> un = A.s0[o];
            A.s2[o] = cadd(A.s2[o], cscale(ku[cc], h / T(3)));
            A.s3[o] = cadd(un, cscale(ku[cc], MODE == UPD_RK4_2 ? h / T(2) : h));
          }
        }
      }
    }
  }
  if (flags) atomicOr(A.status, flags);
}

// ------------------------------------------------------------------------------------------
// z passes (contiguous axis): one thread group of NTZ threads per row unit, inside one warp
// ------------------------------------------------------------------------------------------
// Exchange barrier of the z passes: warp-level when the row units of a warp lie inside it (a row
// per warp at N >= 256; at N = 64 and 128 four and two rows per warp, every lane of the warp
// taking part in every exchange), block-wide for rows that span warps (mixed-radix lengths) and
// for N <= 32 (where the warp-level form gave wrong results in the fused pass).
template <int N>
using ZSync = typename std::conditional<(Cfg<N>::NTZ == 32 || (N >= 64 && Cfg<N>::P2 && 32 % Cfg<N>::NTZ == 0)),
                                        SyncWarp, SyncBlock>::type;
// Row-buffer slot of element i: the same map as the FFT exchange of the row (sidx with PAD).
template <typename T, int N> struct ZIdx {
  static __device__ __forceinline__ int p(int i) { return sidx<T, N, Cfg<N>::EZ, true>(i); }
};

// Hermitian-extended load of Y[k] = A[k] + i B[k] (k = j + NT m), A/B spectral rows with Kin
// valid coefficients; imaginary parts of k = 0 and k = N/2 are dropped (pocketfft c2r).
template <typename T, int N>
__device__ __forceinline__ void zload_pair(cplx<T>* a, const cplx<T>* A, const cplx<T>* B, int Kin,
                                           int j, T s) {
  constexpr int NT = Cfg<N>::NTZ, E = Cfg<N>::EZ;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int k = j + NT * m;
    T yr = 0, yi = 0;
    if (k == 0 || k == N / 2) {
      if (k < Kin) {
        yr = A[k].x;
        if (B) yi = B[k].x;
      }
    } else if (k < N / 2) {
      if (k < Kin) {
        cplx<T> av = A[k];
        cplx<T> bv = B ? B[k] : czero<cplx<T>>();
        yr = av.x - bv.y;
        yi = av.y + bv.x;
      }
    } else {
      const int kk = N - k;
      if (kk < Kin) {
        cplx<T> av = A[kk];
        cplx<T> bv = B ? B[kk] : czero<cplx<T>>();
        yr = av.x + bv.y;
        yi = bv.x - av.y;
      }
    }
    a[m] = cmk(yr * s, yi * s);
  }
}

// After a forward FFT of (a + i b): split Y into A[k], B[k] for k < Kout (zero for k >= Kval).
// Rows of one warp exchange the mirrored coefficients by shuffles; narrower rows write Y to the
// row buffer first (the caller must have synced the buffer).
template <typename T, int N, class Sync>
__device__ __forceinline__ void zstore_pair(const cplx<T>* a, cplx<T>* sb, cplx<T>* A, cplx<T>* B,
                                            int Kout, int Kval, int j, bool ok, Sync sync) {
  constexpr int NT = Cfg<N>::NTZ, E = Cfg<N>::EZ;
  if (B == nullptr) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int k = j + NT * m;
      if (ok && k < Kout) A[k] = k < Kval ? a[m] : czero<cplx<T>>();
    }
    return;
  }
  if constexpr (NT == 32) {
    // a row per warp: Y[N - k] (Y[0] for k = 0) is register E - 1 - m of lane 32 - j (j > 0), or
    // register (E - m) % E of lane 0 (j = 0), fetched by shuffles instead of through the buffer
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int k = j + NT * m;
      cplx<T> z;
      z.x = __shfl_sync(0xffffffffu, a[E - 1 - m].x, (NT - j) & (NT - 1));
      z.y = __shfl_sync(0xffffffffu, a[E - 1 - m].y, (NT - j) & (NT - 1));
      if (j == 0) z = a[(E - m) % E];
      if (ok && k < Kout) {
        cplx<T> ra = czero<cplx<T>>(), rb = czero<cplx<T>>();
        if (k < Kval) {
          const cplx<T> y = a[m];
          ra = cmk(T(0.5) * (y.x + z.x), T(0.5) * (y.y - z.y));
          rb = cmk(T(0.5) * (y.y + z.y), T(-0.5) * (y.x - z.x));
        }
        A[k] = ra;
        B[k] = rb;
      }
    }
    return;
  }
#pragma unroll
  for (int m = 0; m < E; ++m) sb[ZIdx<T, N>::p(j + NT * m)] = a[m];
  sync();
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int k = j + NT * m;
    if (ok && k < Kout) {
      cplx<T> ra = czero<cplx<T>>(), rb = czero<cplx<T>>();
      if (k < Kval) {
        const cplx<T> y = a[m];
        const cplx<T> z = sb[ZIdx<T, N>::p(k == 0 ? 0 : N - k)];
        ra = cmk(T(0.5) * (y.x + z.x), T(0.5) * (y.y - z.y));
        rb = cmk(T(0.5) * (y.y + z.y), T(-0.5) * (y.x - z.x));
      }
      A[k] = ra;
      B[k] = rb;
    }
  }
}

// Generic C2R: pairs of rows (2p, 2p+1) of nrows rows per field; spectral rows of stride ss
// (Kin valid), real rows of stride N.  Scale s (1/N^3 for the 3D inverse).
template <typename T, int N>
__global__ void __launch_bounds__(Cfg<N>::ZTHREADS)
k_z_c2r(const cplx<T>* __restrict__ X, T* __restrict__ x, long long nrows, int ss, int Kin, T s,
        long long xfs, long long Xfs, const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EZ, NT = Cfg<N>::NTZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw);
  const int unit = threadIdx.x / NT, j = threadIdx.x % NT;
  cplx<T>* sb = sbuf + unit * Cfg<N>::ZBUF;
  const long long pair = (long long)blockIdx.x * Cfg<N>::ZROWS + unit;
  const int f = blockIdx.y;
  const bool ok = 2 * pair < nrows;
  const long long r0 = ok ? 2 * pair : 0;
  const cplx<T>* A = X + f * Xfs + r0 * ss;
  const cplx<T>* B = (r0 + 1 < nrows) ? A + ss : nullptr;
  cplx<T> a[E];
  if (ok) zload_pair<T, N>(a, A, B, Kin, j, s);
  else for (int m = 0; m < E; ++m) a[m] = czero<cplx<T>>();
  // the row buffer is private to this unit (one warp or part of one): warp-level sync suffices
  fft_run<T, N, E, true, true>(a, sb, 1, j, tw, ZSync<N>());
  if (!ok) return;
  T* xa = x + f * xfs + r0 * N;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = j + NT * m;
    xa[n] = a[m].x;
    if (B) xa[N + n] = a[m].y;
  }
}

// Generic R2C: pairs of real rows -> spectral rows (stride ss), Kout stored (zeros for k >= Kval).
template <typename T, int N>
__global__ void __launch_bounds__(Cfg<N>::ZTHREADS)
k_z_r2c(const T* __restrict__ x, cplx<T>* __restrict__ X, long long nrows, int ss, int Kout,
        int Kval, long long xfs, long long Xfs, const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EZ, NT = Cfg<N>::NTZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw);
  const int unit = threadIdx.x / NT, j = threadIdx.x % NT;
  cplx<T>* sb = sbuf + unit * Cfg<N>::ZBUF;
  const long long pair = (long long)blockIdx.x * Cfg<N>::ZROWS + unit;
  const int f = blockIdx.y;
  const bool ok = 2 * pair < nrows;
  const long long r0 = ok ? 2 * pair : 0;
  const bool hasb = r0 + 1 < nrows;
  const T* xa = x + f * xfs + r0 * N;
  cplx<T> a[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = j + NT * m;
    a[m] = ok ? cmk(xa[n], hasb ? xa[N + n] : T(0)) : czero<cplx<T>>();
  }
  fft_run<T, N, E, false, true>(a, sb, 1, j, tw, ZSync<N>());
  ZSync<N>()();
  cplx<T>* A = X + f * Xfs + r0 * ss;
  zstore_pair<T, N>(a, sb, A, hasb ? A + ss : nullptr, Kout, Kval, j, ok, ZSync<N>());
}

// One row of the fused z pass: C2R of the six y-transformed fields [u, w] (kz < Kin of each row
// pointer in[f]), optional store of physical u, u x w (F:299-301), R2C of the three products
// (kz < Mzp stored, zero beyond Kin) into P + f*fs + row*Mzp.
// HOIST: the three pairs are loaded before the first transform (rows read from global memory:
// one load phase per row instead of three); the pipelined pass reads staged rows and loads each
// pair just before its transform.
template <typename T, int N, bool HOIST = false>
__device__ __forceinline__ void zcross_row(const cplx<T>* const* in, cplx<T>* sb, cplx<T>* P, long long fs,
                                           long long row, T* uphys, int ulayout, int Mzp, int Kin, T s, int j,
                                           const cplx<T>* __restrict__ tw) {
  constexpr int E = Cfg<N>::EZ, NT = Cfg<N>::NTZ;
  using Sy = ZSync<N>;
  cplx<T> p0[E], p1[E], p2[E];
  zload_pair<T, N>(p0, in[0], in[1], Kin, j, s);  // pair (u_x, u_y)
  if constexpr (HOIST) {
    zload_pair<T, N>(p1, in[2], in[3], Kin, j, s);  // pair (u_z, w_x)
    zload_pair<T, N>(p2, in[4], in[5], Kin, j, s);  // pair (w_y, w_z)
  }
  fft_run<T, N, E, true, true>(p0, sb, 1, j, tw, Sy());
  Sy()();
  if constexpr (!HOIST) zload_pair<T, N>(p1, in[2], in[3], Kin, j, s);
  fft_run<T, N, E, true, true>(p1, sb, 1, j, tw, Sy());
  Sy()();
  if constexpr (!HOIST) zload_pair<T, N>(p2, in[4], in[5], Kin, j, s);
  fft_run<T, N, E, true, true>(p2, sb, 1, j, tw, Sy());
  Sy()();
  if (uphys && ulayout == 0) {  // planar (3, N, N, N)
    const long long NN3 = (long long)N * N * N;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int n = j + NT * m;
      uphys[row * N + n] = p0[m].x;
      uphys[NN3 + row * N + n] = p0[m].y;
      uphys[2 * NN3 + row * N + n] = p1[m].x;
    }
  } else if (uphys) {  // interleaved (N, N, N, 4): (u, v, w, 0) per grid point
    vec4<T>* u4 = reinterpret_cast<vec4<T>*>(uphys);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int n = j + NT * m;
      u4[row * N + n] = mk4<T>(p0[m].x, p0[m].y, p1[m].x, T(0));
    }
  }
  // products: (u x w) = (uy wz - uz wy, uz wx - ux wz, ux wy - uy wx)
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const T ux = p0[m].x, uy = p0[m].y, uz = p1[m].x, wx = p1[m].y, wy = p2[m].x, wz = p2[m].y;
    p0[m] = cmk(wz * uy - wy * uz, wx * uz - wz * ux);
    p1[m] = cmk(wy * ux - wx * uy, T(0));
  }
  fft_run<T, N, E, false, true>(p0, sb, 1, j, tw, Sy());
  Sy()();
  zstore_pair<T, N>(p0, sb, P + row * Mzp, P + fs + row * Mzp, Mzp, Kin, j, true, Sy());
  Sy()();
  fft_run<T, N, E, false, true>(p1, sb, 1, j, tw, Sy());
  zstore_pair<T, N>(p1, sb, P + 2 * fs + row * Mzp, (cplx<T>*)nullptr, Mzp, Kin, j, true, Sy());
}

// Fused z pass, one row unit per NTZ threads, rows read straight from global memory.
// W: (6, N*N, Mzp) in; P: (3, N*N, Mzp) out.
// 64-point FP32 rows (the ensemble's boxes): three CTAs per SM (80 registers, no spills; 86 and
// two CTAs per SM without the bound: ensemble step 1.50 -> 1.42 ms)
template <typename T, int N>
__global__ void __launch_bounds__(Cfg<N>::ZTHREADS, (sizeof(T) == 4 && N == 64) ? 3 : 1)
k_z_cross(const cplx<T>* __restrict__ W, cplx<T>* __restrict__ P, T* __restrict__ uphys, int ulayout, int Mzp,
          int kc, T s, const cplx<T>* __restrict__ tw, long long NR) {
  constexpr int NT = Cfg<N>::NTZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw);
  const int unit = threadIdx.x / NT, j = threadIdx.x % NT;
  cplx<T>* sb = sbuf + unit * Cfg<N>::ZBUF;
  const long long row = (long long)blockIdx.x * Cfg<N>::ZROWS + unit;  // grid covers NR (rows per field) exactly
  (void)Mzp;
  (void)kc;
  constexpr int MZ = Cfg<N>::MZP, KIN = Cfg<N>::KC + 1;  // the plan's cube (checked at launch)
  const long long fs = NR * MZ;
  const cplx<T>* in[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) in[f] = W + f * fs + row * MZ;
  zcross_row<T, N, true>(in, sb, P, fs, row, uphys, ulayout, MZ, KIN, s, j, tw);
}

// Pipelined fused z pass for one warp per row (N >= 256): persistent warps walk the rows with a
// stride; lane 0 of each warp prefetches the next row's six field rows into a double-buffered
// shared staging area with bulk asynchronous copies (the TMA engine), completed on per-buffer
// mbarriers, while the warp transforms the current row.  Waits are bounded: a wait for a row
// gives up after wait_limit polls (the plan's setting); the warp then raises
// LD_STATUS_WAIT_TIMEOUT, drains its copies in flight (bounded by kWaitLimit) and returns.  With
// `stall` set (a test of that path) each warp first waits on a third mbarrier that nothing
// completes, so the wait runs out while the warp's first copy is in flight.
// Shared memory per warp: 2 x 6 x Mzp staging + ZBUF exchange elements, then 3 mbarriers.
constexpr unsigned kWaitLimit = 1u << 24;

// FP32: 8 warps per CTA, two CTAs per SM at N = 256 (at most 128 registers; the 16-element rows
// of N = 512 need more); FP64: 4 warps per CTA
template <typename T, int N>
__global__ void __launch_bounds__(sizeof(T) == 4 ? 256 : 128, (sizeof(T) == 4 && N <= 256) ? 2 : 1)
k_z_cross_pipe(const cplx<T>* __restrict__ W, cplx<T>* __restrict__ P, T* __restrict__ uphys, int ulayout, int Mzp,
               int kc, T s, const cplx<T>* __restrict__ tw, unsigned* status, unsigned wait_limit,
               int stall, long long NR) {
  static_assert(Cfg<N>::NTZ == 32, "one warp per row");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  (void)Mzp;
  (void)kc;
  constexpr int MZ = Cfg<N>::MZP, KIN = Cfg<N>::KC + 1;  // the plan's cube (checked at launch)
  const long long stage_elems = 12LL * MZ;
  cplx<T>* base = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* stage = base + warp * stage_elems;
  cplx<T>* sb = base + nwarps * stage_elems + warp * Cfg<N>::ZBUF;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + nwarps * (stage_elems + Cfg<N>::ZBUF)) + 3 * warp;
  const long long fs = NR * MZ;
  const unsigned rowbytes = (unsigned)(MZ * sizeof(cplx<T>));
  const long long stride = (long long)gridDim.x * nwarps;
  long long row = (long long)blockIdx.x * nwarps + warp;
  if (lane == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], 1);
    mbar_init_fence();
  }
  __syncwarp();
  auto issue = [&](long long r, int b) {
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bars[b], 6u * rowbytes);
#pragma unroll
      for (int f = 0; f < 6; ++f) bulk_g2s(stage + (6 * b + f) * (long long)MZ, W + f * fs + r * MZ, rowbytes, &bars[b]);
    }
  };
  unsigned ph[2] = {0u, 0u};
  bool pend[2] = {false, false};
  if (row < NR) { issue(row, 0); pend[0] = true; }
  if (stall && row < NR && !mbar_wait_bounded(&bars[2], 0u, wait_limit)) {
    if (lane == 0) atomicOr(status, LD_STATUS_WAIT_TIMEOUT);
    mbar_wait_bounded(&bars[0], ph[0], kWaitLimit);  // the first row's copy is in flight
    return;
  }
  int b = 0;
  for (; row < NR; row += stride, b ^= 1) {
    const long long next = row + stride;
    if (next < NR) { issue(next, b ^ 1); pend[b ^ 1] = true; }
    if (!mbar_wait_bounded(&bars[b], ph[b], wait_limit)) {
      if (lane == 0) atomicOr(status, LD_STATUS_WAIT_TIMEOUT);
      for (int q = 0; q < 2; ++q)
        if (pend[q]) mbar_wait_bounded(&bars[q], ph[q], kWaitLimit);
      return;
    }
    ph[b] ^= 1u;
    pend[b] = false;
    const cplx<T>* st = stage + 6 * b * (long long)MZ;
    const cplx<T>* in[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) in[f] = st + f * MZ;
    zcross_row<T, N>(in, sb, P, fs, row, uphys, ulayout, MZ, KIN, s, lane, tw);
    __syncwarp();  // every lane is done with staging buffer b and the exchange buffer
  }
}

// ------------------------------------------------------------------------------------------
// cube <-> reference layout, spectra, forcing, epilogue
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_to_cube(const cplx<T>* __restrict__ full, cplx<T>* __restrict__ cube, int N, int kc,
                          int My, int Mzp, long long total) {
  const int Nf = N / 2 + 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long per = (long long)My * My * Mzp;
    const int comp = (int)(e / per);
    long long r = e - comp * per;
    const int ix = (int)(r / ((long long)My * Mzp));
    r -= (long long)ix * My * Mzp;
    const int iy = (int)(r / Mzp);
    const int kz = (int)(r - (long long)iy * Mzp);
    const int kx = cfreq(ix, kc), ky = cfreq(iy, kc);
    const int k2 = kx * kx + ky * ky + kz * kz;
    cplx<T> v = czero<cplx<T>>();
    if (kz <= kc && k2 <= kc * kc + kc) {
      const int nx = kx < 0 ? kx + N : kx, ny = ky < 0 ? ky + N : ky;
      v = full[(long long)comp * N * N * Nf + ((long long)nx * N + ny) * Nf + kz];
    }
    cube[e] = v;
  }
}

template <typename T>
__global__ void k_from_cube(const cplx<T>* __restrict__ cube, cplx<T>* __restrict__ full, int N, int kc,
                            int My, int Mzp, long long total) {
  const int Nf = N / 2 + 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long per = (long long)N * N * Nf;
    const int comp = (int)(e / per);
    long long r = e - comp * per;
    const int nx = (int)(r / ((long long)N * Nf));
    r -= (long long)nx * N * Nf;
    const int ny = (int)(r / Nf);
    const int kz = (int)(r - (long long)ny * Nf);
    const int ix = crow(nx, N, kc), iy = crow(ny, N, kc);
    cplx<T> v = czero<cplx<T>>();
    if (ix >= 0 && iy >= 0 && kz <= kc)
      v = cube[(long long)comp * My * My * Mzp + ((long long)ix * My + iy) * Mzp + kz];
    full[e] = v;
  }
}

// Shell sums of 0.5 |u|^2 normalize over the modes listed for each shell (CSR of cube indices);
// one CTA per shell, fixed-order FP64 reduction (deterministic).  With `factor` != nullptr the
// block writes the constant-power factor f0 / (2 E_s) of F:250-254 instead of E_s.
template <typename T>
__global__ void k_shell_sum(const cplx<T>* __restrict__ u, long long cs, const int* __restrict__ off,
                            const int* __restrict__ idx, int Mzp, int shell0,
                            double norm0, double* __restrict__ out, double f0, int as_factor, long long ubs = 0,
                            int obs = 0) {
  __shared__ double red[256];
  u += blockIdx.y * ubs;  // box of a multi-box plan
  out += blockIdx.y * obs;
  const int s = shell0 + blockIdx.x;
  double acc = 0.0;
  for (int t = off[s] + threadIdx.x; t < off[s + 1]; t += blockDim.x) {
    const int e = idx[t];
    const double w = (e % Mzp) ? 2.0 : 1.0;  // Hermitian weight of F:136 (kz < N/2 here)
    double m = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cplx<T> v = u[c * cs + e];
      m += double(v.x) * double(v.x) + double(v.y) * double(v.y);
    }
    acc += 0.5 * m * w * norm0;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double e = red[0];
    if (as_factor) {
      if (fabs(e) < 1e-10) e = INFINITY;  // F:250
      out[s] = f0 / (2.0 * e);
    } else {
      out[s] = e;
    }
  }
}

// End-of-step epilogue (F:596-620) on the cube: symmetrise kz = 0 (the irfft->rfft round trip),
// div-free projection, NaN and blow-up tests.  One thread per (kx, ky, kz) column element; the
// kz = 0 pair (k, -k) is handled by the lexicographically smaller member.
template <typename T>
__global__ void k_epilogue(cplx<T>* __restrict__ u, long long cs, int kc, int My, int Mzp,
                           T blowup, unsigned* status) {
  u += blockIdx.y * 3 * cs;  // box of a multi-box plan
  const long long total = (long long)My * My * Mzp;
  unsigned flags = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / ((long long)My * Mzp));
    const long long r = e - (long long)ix * My * Mzp;
    const int iy = (int)(r / Mzp);
    const int kz = (int)(r - (long long)iy * Mzp);
    const int kx = cfreq(ix, kc), ky = cfreq(iy, kc);
    cplx<T> v[3];
    if (kz == 0) {
      // partner -k
      const int jx = kx == 0 ? 0 : (-kx < 0 ? -kx + 2 * kc + 1 : -kx);
      const int jy = ky == 0 ? 0 : (-ky < 0 ? -ky + 2 * kc + 1 : -ky);
      const bool mine = (kx > 0) || (kx == 0 && ky >= 0);
      if (!mine) continue;
      const long long ep = ((long long)jx * My + jy) * Mzp;
      cplx<T> w[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cplx<T> a = u[c * cs + e], b = u[c * cs + ep];
        v[c] = cmk(T(0.5) * (a.x + b.x), T(0.5) * (a.y - b.y));
        w[c] = cconj(v[c]);
      }
      // project both members with their own k
      for (int side = 0; side < 2; ++side) {
        cplx<T>* q = side ? w : v;
        const T qx = T(side ? -kx : kx), qy = T(side ? -ky : ky);
        const int k2 = kx * kx + ky * ky;
        if (k2 > 0 && k2 <= kc * kc + kc) {
          cplx<T> kd = cscale(cadd(cscale(q[0], qx), cscale(q[1], qy)), T(1) / T(k2));
          q[0] = csub(q[0], cscale(kd, qx));
          q[1] = csub(q[1], cscale(kd, qy));
        }
        if (k2 > kc * kc + kc) { q[0] = q[1] = q[2] = czero<cplx<T>>(); }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u[c * cs + e] = v[c];
        if (ep != e) u[c * cs + ep] = w[c];
        if (!(isfinite(v[c].x) && isfinite(v[c].y))) flags |= LD_STATUS_NONFINITE;
        if (v[c].x > blowup || w[c].x > blowup) flags |= LD_STATUS_BLOWUP;
      }
      continue;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = u[c * cs + e];
    const int k2 = kx * kx + ky * ky + kz * kz;
    if (kz <= kc && k2 <= kc * kc + kc) {
      const T qx = T(kx), qy = T(ky), qz = T(kz);
      cplx<T> kd = cscale(cadd(cadd(cscale(v[0], qx), cscale(v[1], qy)), cscale(v[2], qz)), T(1) / T(k2));
      v[0] = csub(v[0], cscale(kd, qx));
      v[1] = csub(v[1], cscale(kd, qy));
      v[2] = csub(v[2], cscale(kd, qz));
    } else {
      v[0] = v[1] = v[2] = czero<cplx<T>>();
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u[c * cs + e] = v[c];
      if (!(isfinite(v[c].x) && isfinite(v[c].y))) flags |= LD_STATUS_NONFINITE;
      if (v[c].x > blowup) flags |= LD_STATUS_BLOWUP;
    }
  }
  if (flags) atomicOr(status, flags);
}

// The step epilogue on the kz = 0 plane only (k_epilogue's kz = 0 branch): for a state whose
// kz > 0 modes the final update stage has already projected and checked.
template <typename T>
__global__ void k_epilogue_plane0(cplx<T>* __restrict__ u, long long cs, int kc, int My, int Mzp, T blowup,
                                  unsigned* status) {
  u += blockIdx.y * 3 * cs;  // box of a multi-box plan
  const long long total = (long long)My * My;
  unsigned flags = 0;
  for (long long e2 = blockIdx.x * (long long)blockDim.x + threadIdx.x; e2 < total; e2 += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e2 / My), iy = (int)(e2 - (long long)ix * My);
    const int kx = cfreq(ix, kc), ky = cfreq(iy, kc);
    const long long e = e2 * Mzp;
    const int jx = kx == 0 ? 0 : (-kx < 0 ? -kx + 2 * kc + 1 : -kx);
    const int jy = ky == 0 ? 0 : (-ky < 0 ? -ky + 2 * kc + 1 : -ky);
    const bool mine = (kx > 0) || (kx == 0 && ky >= 0);
    if (!mine) continue;
    const long long ep = ((long long)jx * My + jy) * Mzp;
    cplx<T> v[3], w[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cplx<T> a = u[c * cs + e], b = u[c * cs + ep];
      v[c] = cmk(T(0.5) * (a.x + b.x), T(0.5) * (a.y - b.y));
      w[c] = cconj(v[c]);
    }
    for (int side = 0; side < 2; ++side) {
      cplx<T>* q = side ? w : v;
      const T qx = T(side ? -kx : kx), qy = T(side ? -ky : ky);
      const int k2 = kx * kx + ky * ky;
      if (k2 > 0 && k2 <= kc * kc + kc) {
        cplx<T> kd = cscale(cadd(cscale(q[0], qx), cscale(q[1], qy)), T(1) / T(k2));
        q[0] = csub(q[0], cscale(kd, qx));
        q[1] = csub(q[1], cscale(kd, qy));
      }
      if (k2 > kc * kc + kc) { q[0] = q[1] = q[2] = czero<cplx<T>>(); }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u[c * cs + e] = v[c];
      if (ep != e) u[c * cs + ep] = w[c];
      if (!(isfinite(v[c].x) && isfinite(v[c].y))) flags |= LD_STATUS_NONFINITE;
      if (v[c].x > blowup || w[c].x > blowup) flags |= LD_STATUS_BLOWUP;
    }
  }
  if (flags) atomicOr(status, flags);
}

template <typename T>
__global__ void k_ifac(T* __restrict__ tab, int n, double nuh) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    tab[i] = T(exp(-nuh * double(i)));
}

// ------------------------------------------------------------------------------------------
// droplets
// ------------------------------------------------------------------------------------------
// Stencil along one axis: base index (periodic) and weights for offsets (lo .. lo+W-1).
template <typename T, int METHOD> struct AxisW;

template <typename T> struct AxisW<T, LD_INTERP_TRILINEAR> {
  static constexpr int W = 2, LO = 0;
  __device__ __forceinline__ static void get(double p, int N, double L, int& i0, T* w) {
    const double s = p * (double(N) / L);
    double fl = floor(s);
    const double t = s - fl;
    long long ii = (long long)fl % N;
    if (ii < 0) ii += N;
    i0 = int(ii);
    w[0] = T(1.0 - t);
    w[1] = T(t);
  }
};

template <typename T> struct AxisW<T, LD_INTERP_TRICUBIC> {
  static constexpr int W = 4, LO = -1;
  __device__ __forceinline__ static void get(double p, int N, double L, int& i0, T* w) {
    const double s = p * (double(N) / L);
    double fl = floor(s);
    const double t = s - fl;
    long long ii = (long long)fl % N;
    if (ii < 0) ii += N;
    i0 = int(ii);
    w[0] = T(-t * (t - 1.0) * (t - 2.0) / 6.0);
    w[1] = T((t + 1.0) * (t - 1.0) * (t - 2.0) / 2.0);
    w[2] = T(-(t + 1.0) * t * (t - 2.0) / 2.0);
    w[3] = T((t + 1.0) * t * (t - 1.0) / 6.0);
  }
};

// The reference's cosine kernel (P:9-16, P:441, P:456): offsets -1..2 around floor(pos/dx),
// weight (1 + cos((pos - X_j) pi / (2 dx))) / 4 with X_j on the periodic index.
template <typename T> struct AxisW<T, LD_INTERP_COSINE> {
  static constexpr int W = 4, LO = -1;
  __device__ __forceinline__ static void get(double p, int N, double L, int& i0, T* w) {
    const double dx = L / double(N);
    const double pm = p - L * floor(p / L);
    long long ii = (long long)floor(pm / dx);
    ii %= N;
    if (ii < 0) ii += N;
    i0 = int(ii);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      int jx = (i0 - 1 + a) % N;
      if (jx < 0) jx += N;
      const double Xj = double(jx) * dx;
      w[a] = T((1.0 + cos((pm - Xj) * (3.14159265358979323846 / (2.0 * dx)))) / 4.0);
    }
  }
};

// i in [-N, 2N) -> i mod N (stencil offsets around a cell index in [0, N); any N)
__device__ __forceinline__ int wrap_index(int i, int N) {
  i = i < 0 ? i + N : i;
  return i >= N ? i - N : i;
}

template <typename T, int METHOD>
__device__ __forceinline__ void gather_point(const T* __restrict__ f, int ncomp, long long fstride, int N,
                                             double L, double px, double py, double pz, T* out) {
  using A = AxisW<T, METHOD>;
  constexpr int W = A::W, LO = A::LO;
  int ix, iy, iz;
  T wx[W], wy[W], wz[W];
  A::get(px, N, L, ix, wx);
  A::get(py, N, L, iy, wy);
  A::get(pz, N, L, iz, wz);
  int jz[W];
#pragma unroll
  for (int c = 0; c < W; ++c) jz[c] = wrap_index(iz + LO + c, N);
  for (int c = 0; c < ncomp; ++c) out[c] = T(0);
#pragma unroll
  for (int a = 0; a < W; ++a) {
    const int jx = wrap_index(ix + LO + a, N);
#pragma unroll
    for (int b = 0; b < W; ++b) {
      const int jy = wrap_index(iy + LO + b, N);
      const long long base = ((long long)jx * N + jy) * N;
      const T wab = wx[a] * wy[b];
      for (int c = 0; c < ncomp; ++c) {
        const T* fc = f + c * fstride + base;
        T acc = T(0);
#pragma unroll
        for (int q = 0; q < W; ++q) acc += wz[q] * __ldg(fc + jz[q]);
        out[c] += wab * acc;
      }
    }
  }
}

template <typename T, int METHOD>
__global__ void k_gather(const T* __restrict__ f, int ncomp, int N, double L, const double* __restrict__ pos,
                         long long n, T* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T v[8];
    gather_point<T, METHOD>(f, ncomp, (long long)N * N * N, N, L, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], v);
    for (int c = 0; c < ncomp; ++c) out[i * ncomp + c] = v[c];
  }
}

// Interpolation of an interleaved (N, N, N, 4) velocity: one 16/32-byte load per stencil point.
template <typename T, int METHOD>
__device__ __forceinline__ void gather_point4(const vec4<T>* __restrict__ f, int N, double L, double px, double py,
                                              double pz, T* out) {
  using A = AxisW<T, METHOD>;
  constexpr int W = A::W, LO = A::LO;
  int ix, iy, iz;
  T wx[W], wy[W], wz[W];
  A::get(px, N, L, ix, wx);
  A::get(py, N, L, iy, wy);
  A::get(pz, N, L, iz, wz);
  int jz[W];
#pragma unroll
  for (int c = 0; c < W; ++c) jz[c] = wrap_index(iz + LO + c, N);
  T o0 = 0, o1 = 0, o2 = 0;
#pragma unroll
  for (int a = 0; a < W; ++a) {
    const int jx = wrap_index(ix + LO + a, N);
#pragma unroll
    for (int b = 0; b < W; ++b) {
      const int jy = wrap_index(iy + LO + b, N);
      const vec4<T>* row = f + ((long long)jx * N + jy) * N;
      T s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        const vec4<T> v = row[jz[q]];
        s0 += wz[q] * v.x;
        s1 += wz[q] * v.y;
        s2 += wz[q] * v.z;
      }
      const T wab = wx[a] * wy[b];
      o0 += wab * s0;
      o1 += wab * s1;
      o2 += wab * s2;
    }
  }
  out[0] = o0;
  out[1] = o1;
  out[2] = o2;
}

template <typename T, int METHOD>
__global__ void k_gather4(const vec4<T>* __restrict__ f, int N, double L, const double* __restrict__ pos, long long n,
                          T* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T v[3];
    gather_point4<T, METHOD>(f, N, L, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], v);
    out[3 * i] = v[0];
    out[3 * i + 1] = v[1];
    out[3 * i + 2] = v[2];
  }
}

template <typename T, int METHOD, int STAGE>
__global__ void k_droplet_stage(const vec4<T>* __restrict__ u0, int N, double L, double* __restrict__ pos,
                                T* __restrict__ vel, const T* __restrict__ tau, T* __restrict__ a1,
                                long long n, double h, T g, const int* __restrict__ box = nullptr) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    // the droplet's box of a multi-box plan: its field is box (N, N, N, 4) further on
    const vec4<T>* u = box ? u0 + (long long)box[i] * N * N * N : u0;
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const T vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
    const T it = T(1) / tau[i];
    T up[3];
    if (STAGE == 1) {
      gather_point4<T, METHOD>(u, N, L, px, py, pz, up);
      a1[3 * i] = (up[0] - vx) * it;
      a1[3 * i + 1] = (up[1] - vy) * it;
      a1[3 * i + 2] = (up[2] - vz) * it - g;
    } else {
      const T ax = a1[3 * i], ay = a1[3 * i + 1], az = a1[3 * i + 2];
      const T hh = T(h);
      const T sx = vx + hh * ax, sy = vy + hh * ay, sz = vz + hh * az;  // vs = v + h a1
      const double qx = px + h * double(vx), qy = py + h * double(vy), qz = pz + h * double(vz);
      gather_point4<T, METHOD>(u, N, L, qx, qy, qz, up);
      const T bx = (up[0] - sx) * it, by = (up[1] - sy) * it, bz = (up[2] - sz) * it - g;
      pos[3 * i] = px + 0.5 * h * (double(vx) + double(sx));
      pos[3 * i + 1] = py + 0.5 * h * (double(vy) + double(sy));
      pos[3 * i + 2] = pz + 0.5 * h * (double(vz) + double(sz));
      vel[3 * i] = vx + T(0.5) * hh * (ax + bx);
      vel[3 * i + 1] = vy + T(0.5) * hh * (ay + by);
      vel[3 * i + 2] = vz + T(0.5) * hh * (az + bz);
    }
  }
}

}  // namespace ld
