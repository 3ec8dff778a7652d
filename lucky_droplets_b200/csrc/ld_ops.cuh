// Launch sequences for one (precision, N) instance.  Included by the ld_inst_*.cu units, each
// of which instantiates one OpsTable; compiling the twelve instances separately keeps the build
// parallel.
#pragma once
#include <cmath>
#include <type_traits>

#include "ld_internal.cuh"
#include "ld_kernels.cuh"

namespace ld_impl {

using namespace ld;

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

template <class K> int set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) { ld_set_last_error(e); return LD_ERR_CUDA; }
  }
  return LD_OK;
}

inline long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

inline int grid1d(long long n, int threads) {
  long long b = cdiv(n, threads);
  if (b > 148LL * 32) b = 148LL * 32;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename T, int N> struct Ops {
  using C = cplx<T>;
  static constexpr int TB = Cfg<N>::TB;
  static constexpr size_t COL_SMEM = sizeof(C) * N * TB;
  static constexpr size_t Z_SMEM = sizeof(C) * Cfg<N>::ZROWS * Cfg<N>::ZBUF;

  template <bool INV, class Ld, class St>
  static int colpass(ld_plan* p, int kid, Ld ld, St st, int ncols, int nf, int nouter, const C* tw, cudaStream_t s) {
    ProfScope ps(p, kid, s);
    auto k = colfft_kernel<T, N, INV, Ld, St>();
    if (int rc = set_smem(k, COL_SMEM)) return rc;
    dim3 grid((unsigned)(cdiv(ncols, TB) * nf), (unsigned)nouter);
    k<<<grid, Cfg<N>::COL_THREADS, COL_SMEM, s>>>(ld, st, ncols, nf, tw);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  // Column pass over plain strided rows: the pipelined kernel where two staging buffers fit.
  static constexpr bool PIPE = 2 * COL_SMEM <= 72 * 1024;
  // IN_MAP: the input rows are compact cube rows (in.kc >= 0), fixed at compile time for the
  // pipelined kernel
  template <bool INV, bool IN_MAP, class St>
  static int colpass_rows(ld_plan* p, int kid, RowsIO<T> in, St st, int ncols, int nf, int nouter, const C* tw,
                          cudaStream_t s, int variant = -2) {
    const int choice = variant != -2 ? variant : p->tune_y[INV ? 0 : 1];
    if constexpr (!PIPE) {
      return colpass<INV>(p, kid, LdRowsC<T, N, IN_MAP>{in}, st, ncols, nf, nouter, tw, s);
    } else {
      if (choice == 0 || cdiv(ncols, TB) * (long long)nf * nouter >= (1LL << 31))
        return colpass<INV>(p, kid, LdRowsC<T, N, IN_MAP>{in}, st, ncols, nf, nouter, tw, s);
      ProfScope ps(p, kid, s);
      auto k = k_colfft_pipe<T, N, INV, St, IN_MAP>;
      if (int rc = set_smem(k, 2 * COL_SMEM)) return rc;
      static int occ = 0;
      if (occ == 0) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, Cfg<N>::COL_THREADS, 2 * COL_SMEM);
        if (e != cudaSuccess || occ < 1) occ = 1;
      }
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const long long items = cdiv(ncols, TB) * (long long)nf * nouter;
      const int per_sm = choice > 0 && choice < occ ? choice : occ;
      const long long grid = items < (long long)sms * per_sm ? items : (long long)sms * per_sm;
      k<<<(unsigned)grid, Cfg<N>::COL_THREADS, 2 * COL_SMEM, s>>>(in, st, ncols, nf, nouter, tw);
      LD_LAUNCH_CHECK();
      return LD_OK;
    }
  }

  static RowsIO<T> io(const void* p, long long fs, long long os, int rs, int kc) {
    RowsIO<T> r;
    r.p = (C*)p; r.fs = fs; r.os = os; r.rs = rs; r.kc = kc;
    return r;
  }

  static int z_c2r(ld_plan* p, const C* X, T* x, long long nrows, int ss, int Kin, T sc, long long xfs, long long Xfs,
                   int nf, const C* tw, cudaStream_t s) {
    ProfScope ps(p, KID_ZC2R, s);
    auto k = k_z_c2r<T, N>;
    if (int rc = set_smem(k, Z_SMEM)) return rc;
    dim3 grid((unsigned)cdiv(nrows / 2, Cfg<N>::ZROWS), (unsigned)nf);
    k<<<grid, Cfg<N>::ZTHREADS, Z_SMEM, s>>>(X, x, nrows, ss, Kin, sc, xfs, Xfs, tw);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  static int z_r2c(ld_plan* p, const T* x, C* X, long long nrows, int ss, int Kout, int Kval, long long xfs, long long Xfs,
                   int nf, const C* tw, cudaStream_t s) {
    ProfScope ps(p, KID_ZR2C, s);
    auto k = k_z_r2c<T, N>;
    if (int rc = set_smem(k, Z_SMEM)) return rc;
    dim3 grid((unsigned)cdiv(nrows / 2, Cfg<N>::ZROWS), (unsigned)nf);
    k<<<grid, Cfg<N>::ZTHREADS, Z_SMEM, s>>>(x, X, nrows, ss, Kout, Kval, xfs, Xfs, tw);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  // ---- reference-layout transforms --------------------------------------------------------
  static int rfft_full(ld_plan* p, const T* u, C* fu, int ncomp, cudaStream_t s) {
    const int Nf = p->Nf;
    const C* tw = (const C*)p->tw;
    const long long NN = (long long)N * N;
    if (int rc = z_r2c(p, u, fu, NN, Nf, Nf, Nf, NN * N, NN * Nf, ncomp, tw, s)) return rc;
    // y pass in place: columns kz (Nf), rows y, outer x
    auto yio = io(fu, NN * Nf, (long long)N * Nf, Nf, -1);
    if (int rc = colpass<false>(p, KID_YFWD, LdRowsC<T, N, false>{yio}, StRowsC<T, N, false>{yio}, Nf, ncomp, N, tw, s)) return rc;
    // x pass in place: columns (ky, kz) flat, rows x
    auto xio = io(fu, NN * Nf, 0, N * Nf, -1);
    return colpass<false>(p, KID_XPASS, LdRowsC<T, N, false>{xio}, StRowsC<T, N, false>{xio}, N * Nf, ncomp, 1, tw, s);
  }

  static int irfft_full(ld_plan* p, const C* fu, T* u, int ncomp, cudaStream_t s) {
    const int Nf = p->Nf;
    const C* tw = (const C*)p->tw;
    const long long NN = (long long)N * N;
    const long long per = NN * Nf;
    const int chunk = (int)(((long long)6 * NN * p->Mzp) / per);  // fields that fit in W2
    C* W = (C*)p->W2;
    for (int c0 = 0; c0 < ncomp; c0 += chunk) {
      const int nc = ncomp - c0 < chunk ? ncomp - c0 : chunk;
      auto xin = io(fu + c0 * per, per, 0, N * Nf, -1);
      auto xout = io(W, per, 0, N * Nf, -1);
      if (int rc = colpass<true>(p, KID_XPASS, LdRowsC<T, N, false>{xin}, StRowsC<T, N, false>{xout}, N * Nf, nc, 1, tw, s)) return rc;
      auto yio = io(W, per, (long long)N * Nf, Nf, -1);
      if (int rc = colpass<true>(p, KID_YINV, LdRowsC<T, N, false>{yio}, StRowsC<T, N, false>{yio}, Nf, nc, N, tw, s)) return rc;
      const T sc = T(1.0 / (double(N) * N * N));
      if (int rc = z_c2r(p, W, u + (long long)c0 * NN * N, NN, Nf, Nf, sc, NN * N, per, nc, tw, s)) return rc;
    }
    return LD_OK;
  }

  // ---- cube-layout (dealiased) transforms -----------------------------------------------------
  static int irfft_cube(ld_plan* p, const C* uk, T* u, int ncomp, cudaStream_t s) {
    const int kc = p->kc, My = p->My, Mzp = p->Mzp;
    const C* tw = (const C*)p->tw;
    const long long NN = (long long)N * N;
    const long long cs = p->cube_elems();
    C* W1 = (C*)p->W1;
    C* W2 = (C*)p->W2;
    const long long w1s = (long long)N * My * Mzp, w2s = NN * Mzp;
    for (int c0 = 0; c0 < ncomp; c0 += 6) {
      const int nc = ncomp - c0 < 6 ? ncomp - c0 : 6;
      auto xin = io(uk + c0 * cs, cs, 0, My * Mzp, kc);
      auto xout = io(W1, w1s, 0, My * Mzp, -1);
      if (int rc = colpass<true>(p, KID_XPASS, LdRowsC<T, N, true>{xin}, StRowsC<T, N, false>{xout}, My * Mzp, nc, 1, tw, s)) return rc;
      auto yin = io(W1, w1s, (long long)My * Mzp, Mzp, kc);
      auto yout = io(W2, w2s, (long long)N * Mzp, Mzp, -1);
      if (int rc = colpass<true>(p, KID_YINV, LdRowsC<T, N, true>{yin}, StRowsC<T, N, false>{yout}, Mzp, nc, N, tw, s)) return rc;
      const T sc = T(1.0 / (double(N) * N * N));
      if (int rc = z_c2r(p, W2, u + (long long)c0 * NN * N, NN, Mzp, kc + 1, sc, NN * N, w2s, nc, tw, s)) return rc;
    }
    return LD_OK;
  }

  static int rfft_cube(ld_plan* p, const T* u, C* uk, int ncomp, cudaStream_t s) {
    const int kc = p->kc, My = p->My, Mzp = p->Mzp;
    const C* tw = (const C*)p->tw;
    const long long NN = (long long)N * N;
    const long long cs = p->cube_elems();
    C* W1 = (C*)p->W1;
    C* W2 = (C*)p->W2;
    const long long w1s = (long long)N * My * Mzp, w2s = NN * Mzp;
    for (int c0 = 0; c0 < ncomp; c0 += 6) {
      const int nc = ncomp - c0 < 6 ? ncomp - c0 : 6;
      if (int rc = z_r2c(p, u + (long long)c0 * NN * N, W2, NN, Mzp, Mzp, kc + 1, NN * N, w2s, nc, tw, s)) return rc;
      auto yin = io(W2, w2s, (long long)N * Mzp, Mzp, -1);
      auto yout = io(W1, w1s, (long long)My * Mzp, Mzp, kc);
      if (int rc = colpass<false>(p, KID_YFWD, LdRowsC<T, N, false>{yin}, StRowsC<T, N, true>{yout}, Mzp, nc, N, tw, s)) return rc;
      auto xin = io(W1, w1s, 0, My * Mzp, -1);
      auto xout = io(uk + c0 * cs, cs, 0, My * Mzp, kc);
      if (int rc = colpass<false>(p, KID_XPASS, LdRowsC<T, N, false>{xin}, StCube<T, N>{xout, Mzp}, My * Mzp, nc, 1, tw, s)) return rc;
    }
    return LD_OK;
  }

  // ---- forcing factor for the stage input -----------------------------------------------------
  static int forcing_factor(ld_plan* p, const C* y, const ld_flow_params* prm, cudaStream_t s) {
    if (prm->kf_hi < prm->kf_lo || prm->f0 == 0.0) return LD_OK;
    ProfScope ps(p, KID_FORCING, s);
    const double norm0 = std::pow(2.0 * M_PI, 3) / std::pow((double)N, 6);
    dim3 grid((unsigned)(prm->kf_hi - prm->kf_lo + 1), (unsigned)p->nbox);
    k_shell_sum<T><<<grid, 256, 0, s>>>(y, p->cube_elems(), p->shell_off, p->shell_idx, p->Mzp, prm->kf_lo, norm0,
                                        p->factor, prm->f0, 1, 3 * p->cube_elems(), p->Nf);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  // The integrating-factor table exp(-nu h k^2) for the current nu h, built on the stream when
  // nu h changes.  While the stream is being captured into a CUDA graph the table kernel is
  // recorded into the graph and the table is not marked built: the graph may never be replayed
  // (a discarded capture), so only a launch that runs marks it.
  static int ensure_ifac(ld_plan* p, double nuh, cudaStream_t s) {
    if (p->ifac_key == nuh) return LD_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    LD_CUDA_CHECK(cudaStreamIsCapturing(s, &cap));
    ProfScope ps(p, KID_IFAC, s);
    k_ifac<T><<<grid1d(p->nifac, 256), 256, 0, s>>>((T*)p->ifac, p->nifac, nuh);
    LD_LAUNCH_CHECK();
    if (cap == cudaStreamCaptureStatusNone) p->ifac_key = nuh;
    return LD_OK;
  }

  // ---- pipelined fused z pass (one warp per row) -------------------------------------------------
  static int zcross_pipe(ld_plan* p, const C* W2, C* W1, T* uout, int ulayout, T sc, cudaStream_t s) {
    constexpr int WARPS = sizeof(T) == 4 ? 8 : 4;
    const long long NN = (long long)N * N * p->nbox;  // rows per field, all boxes
    const size_t smem = (size_t)WARPS * ((size_t)12 * p->Mzp + Cfg<N>::ZBUF) * sizeof(C) + 24 * WARPS;
    auto k = k_z_cross_pipe<T, N>;
    if (int rc = set_smem(k, smem)) return rc;
    static int blocks_per_sm = -1;
    if (blocks_per_sm < 0) {
      int b = 0;
      cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, WARPS * 32, smem);
      if (e != cudaSuccess) { ld_set_last_error(e); return LD_ERR_CUDA; }
      blocks_per_sm = b > 0 ? b : 1;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long grid = (long long)sms * blocks_per_sm;
    const long long need = (NN + WARPS - 1) / WARPS;
    if (grid > need) grid = need;
    k<<<(unsigned)grid, WARPS * 32, smem, s>>>(W2, W1, uout, ulayout, p->Mzp, p->kc, sc, (const C*)p->tw, p->status,
                                               p->wait_limit, p->wait_stall, NN);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  // ---- autotuner of the y passes: every launch variant timed on the plan's workspace ------------
  static int autotune(ld_plan* p, cudaStream_t s, double* ms) {
    const int My = p->My, Mzp = p->Mzp, kc = p->kc;
    const C* tw = (const C*)p->tw;
    C* W1 = (C*)p->W1;
    C* W2 = (C*)p->W2;
    const long long NN = (long long)N * N, w1s = (long long)N * My * Mzp, w2s = NN * Mzp;
    cudaEvent_t a, b;
    LD_CUDA_CHECK(cudaEventCreate(&a));
    LD_CUDA_CHECK(cudaEventCreate(&b));
    const int nv = PIPE ? 4 : 1;
    for (int pass = 0; pass < 2; ++pass) {
      double best = 1e30;
      int pick = -1;
      for (int v = 0; v < 4; ++v) {
        ms[4 * pass + v] = -1.0;
        if (v >= nv) continue;
        auto run = [&]() -> int {
          const int nb = p->nbox;
          if (pass == 0)
            return colpass_rows<true, true>(p, KID_YINV, io(W1, nb * w1s, (long long)My * Mzp, Mzp, kc),
                                            StRowsC<T, N, false>{io(W2, nb * w2s, (long long)N * Mzp, Mzp, -1)}, Mzp,
                                            6, nb * N, tw, s, v);
          return colpass_rows<false, false>(p, KID_YFWD, io(W1, nb * w2s, (long long)N * Mzp, Mzp, -1),
                                            StRowsC<T, N, true>{io(W2, nb * w1s, (long long)My * Mzp, Mzp, kc)}, Mzp,
                                            3, nb * N, tw, s, v);
        };
        if (int rc = run()) return rc;  // warm-up
        LD_CUDA_CHECK(cudaEventRecord(a, s));
        for (int r = 0; r < 5; ++r)
          if (int rc = run()) return rc;
        LD_CUDA_CHECK(cudaEventRecord(b, s));
        LD_CUDA_CHECK(cudaEventSynchronize(b));
        float t = 0.f;
        LD_CUDA_CHECK(cudaEventElapsedTime(&t, a, b));
        ms[4 * pass + v] = t / 5.0;
        if (t / 5.0 < best) { best = t / 5.0; pick = v; }
      }
      p->tune_y[pass] = PIPE ? pick : 0;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return LD_OK;
  }

  // ---- RHS pipeline: y (stage input) -> update epilogue ------------------------------------------
  template <int MODE>
  static int rhs(ld_plan* p, C* s0, C* s1, C* s2, T* uout, const ld_flow_params* prm, double visc,
                 cudaStream_t s, C* s3 = nullptr) {
    const int kc = p->kc, My = p->My, Mzp = p->Mzp;
    if (kc != Cfg<N>::KC || My != Cfg<N>::MY || Mzp != Cfg<N>::MZP)  // the kernels fix the cube by N
      return ld_fail(LD_ERR_UNSUPPORTED, "plan cube (%d, %d, %d) differs from N = %d's", kc, My, Mzp, N);
    const C* tw = (const C*)p->tw;
    const long long NN = (long long)N * N;
    const long long cs = p->cube_elems();
    C* W1 = (C*)p->W1;
    C* W2 = (C*)p->W2;
    const long long w1s = (long long)N * My * Mzp, w2s = NN * Mzp;
    const C* y = s1;  // stage input in every mode
    // boxes of a multi-box plan: each pass is one launch over all of them; the workspace holds
    // the box index next to x (fields (f, box, x, ...)), so that (box, x) is one outer index
    const int nb = p->nbox;
    if (nb > 1 && p->sm_vk) return ld_fail(LD_ERR_UNSUPPORTED, "slow-manifold output of a multi-box plan");
    if (int rc = forcing_factor(p, y, prm, s)) return rc;
    // inverse x pass with the curl: 6 fields [u, w]
    LdCurl<T, N> lc{y, cs, kc, My, Mzp, 3 * cs};
    auto xout = io(W1, nb * w1s, w1s, My * Mzp, -1);
    if (int rc = colpass<true>(p, KID_XINV, lc, StRowsC<T, N, false>{xout}, My * Mzp, 6, nb, tw, s)) return rc;
    // inverse y pass
    auto yin = io(W1, nb * w1s, (long long)My * Mzp, Mzp, kc);
    auto yout = io(W2, nb * w2s, (long long)N * Mzp, Mzp, -1);
    if (int rc = colpass_rows<true, true>(p, KID_YINV, yin, StRowsC<T, N, false>{yout}, Mzp, 6, nb * N, tw, s))
      return rc;
    // fused z pass: u, w -> u x w  (W2 -> W1 as (3, N*N, Mzp))
    {
      ProfScope ps(p, KID_ZCROSS, s);
      const T sc = T(1.0 / (double(N) * N * N));
      const int ulayout = (MODE == UPD_RHS) ? 0 : 1;  // the time steppers feed droplets: interleaved
      if constexpr (Cfg<N>::NTZ == 32) {
        if (int rc = zcross_pipe(p, W2, W1, uout, ulayout, sc, s)) return rc;
      } else {
        auto k = k_z_cross<T, N>;
        if (int rc = set_smem(k, Z_SMEM)) return rc;
        const long long rows = NN * nb;
        k<<<(unsigned)(rows / Cfg<N>::ZROWS), Cfg<N>::ZTHREADS, Z_SMEM, s>>>(W2, W1, uout, ulayout, Mzp, kc, sc, tw,
                                                                            rows);
        LD_LAUNCH_CHECK();
      }
    }
    // forward y pass (W1 -> W2 as (3, N, My, Mzp))
    auto fyin = io(W1, nb * w2s, (long long)N * Mzp, Mzp, -1);
    auto fyout = io(W2, nb * w1s, (long long)My * Mzp, Mzp, kc);
    if (int rc = colpass_rows<false, false>(p, KID_YFWD, fyin, StRowsC<T, N, true>{fyout}, Mzp, 3, nb * N, tw, s))
      return rc;
    // forward x pass + k-space update
    UpdArgs<T> A;
    A.nl = W2; A.nls = nb * w1s;
    A.nl_bs = w1s; A.cube_bs = 3 * cs; A.fac_bs = p->Nf;
    A.s0 = s0; A.s1 = s1; A.s2 = s2; A.s3 = s3; A.cs = cs;
    A.factor = p->factor; A.kf_lo = prm->kf_lo; A.kf_hi = (prm->f0 == 0.0) ? -1 : prm->kf_hi;
    A.ifac = (const T*)p->ifac;
    A.h = T(prm->dt); A.nu = T(prm->nu); A.visc = T(visc);
    A.kc = kc; A.My = My; A.Mzp = Mzp; A.status = p->status;
    A.vk = (C*)p->sm_vk; A.tps = T(p->sm_tps); A.vg = T(p->sm_tps * p->sm_g * (double)N * N * N);
    A.blowup = T(100.0 * (double)N * N * N);  // the blow-up threshold of the step epilogue (F:618)
    // RK2 stages stage their cube rows in shared memory when that keeps 2 CTAs per SM
    const size_t pre_bytes = sizeof(C) * 3 * (size_t)(2 * kc + 1) * TB;
    constexpr bool RK2 = MODE == UPD_RK2_1 || MODE == UPD_RK2_2;
    A.prefetch = (RK2 && COL_SMEM + pre_bytes <= 112 * 1024) ? 1 : 0;
    const size_t smem = COL_SMEM + (A.prefetch ? pre_bytes : 0);
    ProfScope ps(p, KID_XFWD_UPD, s);
    auto k = k_xfwd_update<T, N, MODE>;
    if (int rc = set_smem(k, smem)) return rc;
    dim3 ugrid((unsigned)cdiv((long long)My * Mzp, TB), (unsigned)nb);
    k<<<ugrid, Cfg<N>::COL_THREADS, smem, s>>>(A, My * Mzp, tw);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  static int gather(ld_plan* p, const T* f, int ncomp, const double* pos, long long n, int method, T* out,
                    cudaStream_t s) {
    ProfScope ps(p, KID_GATHER, s);
    const int th = 256;
    const int g = grid1d(n, th);
    const double L = 2.0 * M_PI;
    if (method == LD_INTERP_TRILINEAR) k_gather<T, LD_INTERP_TRILINEAR><<<g, th, 0, s>>>(f, ncomp, N, L, pos, n, out);
    else if (method == LD_INTERP_TRICUBIC) k_gather<T, LD_INTERP_TRICUBIC><<<g, th, 0, s>>>(f, ncomp, N, L, pos, n, out);
    else k_gather<T, LD_INTERP_COSINE><<<g, th, 0, s>>>(f, ncomp, N, L, pos, n, out);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  template <int M>
  static int dstage_m(ld_plan* p, int stage, const T* u, double* pos, T* vel, const T* tau, T* a1, long long n, double h,
                      double g, const int* box, cudaStream_t s) {
    ProfScope ps(p, stage == 1 ? KID_DROPLET1 : KID_DROPLET2, s);
    const int th = 256;
    const int gr = grid1d(n, th);
    const double L = 2.0 * M_PI;
    const vec4<T>* u4 = reinterpret_cast<const vec4<T>*>(u);
    if (stage == 1) k_droplet_stage<T, M, 1><<<gr, th, 0, s>>>(u4, N, L, pos, vel, tau, a1, n, h, T(g), box);
    else k_droplet_stage<T, M, 2><<<gr, th, 0, s>>>(u4, N, L, pos, vel, tau, a1, n, h, T(g), box);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  static int dstage(ld_plan* p, int stage, int method, const T* u, double* pos, T* vel, const T* tau, T* a1, long long n,
                    double h, double g, const int* box, cudaStream_t s) {
    if (method == LD_INTERP_TRILINEAR)
      return dstage_m<LD_INTERP_TRILINEAR>(p, stage, u, pos, vel, tau, a1, n, h, g, box, s);
    if (method == LD_INTERP_TRICUBIC)
      return dstage_m<LD_INTERP_TRICUBIC>(p, stage, u, pos, vel, tau, a1, n, h, g, box, s);
    return dstage_m<LD_INTERP_COSINE>(p, stage, u, pos, vel, tau, a1, n, h, g, box, s);
  }
};


// ---- type-erased wrappers ------------------------------------------------------------------
template <typename T, int N> struct Table {
  using O = Ops<T, N>;
  using C = ld::cplx<T>;
  static int rfft_full(ld_plan* p, const void* u, void* fu, int nc, cudaStream_t s) {
    return O::rfft_full(p, (const T*)u, (C*)fu, nc, s);
  }
  static int irfft_full(ld_plan* p, const void* fu, void* u, int nc, cudaStream_t s) {
    return O::irfft_full(p, (const C*)fu, (T*)u, nc, s);
  }
  static int irfft_cube(ld_plan* p, const void* uk, void* u, int nc, cudaStream_t s) {
    return O::irfft_cube(p, (const C*)uk, (T*)u, nc, s);
  }
  static int rfft_cube(ld_plan* p, const void* u, void* uk, int nc, cudaStream_t s) {
    return O::rfft_cube(p, (const T*)u, (C*)uk, nc, s);
  }
  static int to_cube(ld_plan* p, const void* full, void* cube, int nc, cudaStream_t s) {
    ProfScope ps(p, KID_CONVERT, s);
    const long long total = p->cube_elems() * nc;
    ld::k_to_cube<T><<<grid1d(total, 256), 256, 0, s>>>((const C*)full, (C*)cube, p->N, p->kc, p->My, p->Mzp, total);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }
  static int from_cube(ld_plan* p, const void* cube, void* full, int nc, cudaStream_t s) {
    ProfScope ps(p, KID_CONVERT, s);
    const long long total = (long long)p->N * p->N * p->Nf * nc;
    ld::k_from_cube<T><<<grid1d(total, 256), 256, 0, s>>>((const C*)cube, (C*)full, p->N, p->kc, p->My, p->Mzp, total);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }
  static int shell_spectrum(ld_plan* p, const void* uk, double* ek, cudaStream_t s) {
    ProfScope ps(p, KID_SHELL, s);
    const double norm0 = std::pow(2.0 * M_PI, 3) / std::pow((double)N, 6);
    ld::k_shell_sum<T><<<p->Nf, 256, 0, s>>>((const C*)uk, p->cube_elems(), p->shell_off, p->shell_idx, p->Mzp, 0,
                                             norm0, ek, 0.0, 0);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }
  static int autotune(ld_plan* p, cudaStream_t s, double* ms) { return O::autotune(p, s, ms); }
  static int prepare(ld_plan* p, const ld_flow_params* prm, cudaStream_t s) {
    return O::ensure_ifac(p, prm->nu * prm->dt, s);
  }
  static int rhs(ld_plan* p, int mode, void* s0, void* s1, void* s2, void* s3, void* uout,
                 const ld_flow_params* prm, double visc, cudaStream_t s) {
    C *a = (C*)s0, *b = (C*)s1, *c = (C*)s2, *d = (C*)s3;
    if (mode == ld::UPD_RK2_1 || mode == ld::UPD_RK2_2)
      if (int rc = O::ensure_ifac(p, prm->nu * prm->dt, s)) return rc;
    switch (mode) {
      case ld::UPD_RHS: return O::template rhs<ld::UPD_RHS>(p, a, b, c, (T*)uout, prm, visc, s, d);
      case ld::UPD_RK2_1: return O::template rhs<ld::UPD_RK2_1>(p, a, b, c, (T*)uout, prm, visc, s, d);
      case ld::UPD_RK2_2: return O::template rhs<ld::UPD_RK2_2>(p, a, b, c, (T*)uout, prm, visc, s, d);
      case ld::UPD_RK4_1: return O::template rhs<ld::UPD_RK4_1>(p, a, b, c, (T*)uout, prm, visc, s, d);
      case ld::UPD_RK4_2: return O::template rhs<ld::UPD_RK4_2>(p, a, b, c, (T*)uout, prm, visc, s, d);
      case ld::UPD_RK4_3: return O::template rhs<ld::UPD_RK4_3>(p, a, b, c, (T*)uout, prm, visc, s, d);
      case ld::UPD_RK4_4: return O::template rhs<ld::UPD_RK4_4>(p, a, b, c, (T*)uout, prm, visc, s, d);
      default: return ld_fail(LD_ERR_ARG, "bad update mode %d", mode);
    }
  }
  static int epilogue(ld_plan* p, void* uk, cudaStream_t s) {
    ProfScope ps(p, KID_EPILOGUE, s);
    const long long total = p->cube_elems();
    const double blow = 100.0 * (double)N * N * N;
    dim3 grid((unsigned)grid1d(total, 256), (unsigned)p->nbox);
    ld::k_epilogue<T><<<grid, 256, 0, s>>>((C*)uk, total, p->kc, p->My, p->Mzp, T(blow), p->status);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }  static int epilogue0(ld_plan* p, void* uk, cudaStream_t s) {
    ProfScope ps(p, KID_EPILOGUE, s);
    const double blow = 100.0 * (double)N * N * N;
    const long long plane = (long long)p->My * p->My;
    dim3 grid((unsigned)grid1d(plane, 256), (unsigned)p->nbox);
    ld::k_epilogue_plane0<T><<<grid, 256, 0, s>>>((C*)uk, p->cube_elems(), p->kc, p->My, p->Mzp, T(blow), p->status);
    LD_LAUNCH_CHECK();
    return LD_OK;
  }

  static int gather(ld_plan* p, const void* f, int nc, const double* pos, long long n, int method, void* out,
                    cudaStream_t s) {
    return O::gather(p, (const T*)f, nc, pos, n, method, (T*)out, s);
  }
  static int dstage(ld_plan* p, int stage, int method, const void* u, double* pos, void* vel, const void* tau,
                    void* a1, long long n, double h, double g, const int* box, cudaStream_t s) {
    return O::dstage(p, stage, method, (const T*)u, pos, (T*)vel, (const T*)tau, (T*)a1, n, h, g, box, s);
  }
  static const OpsTable* get() {
    static const OpsTable t = {rfft_full, irfft_full, irfft_cube, rfft_cube, to_cube, from_cube,
                               shell_spectrum, rhs, epilogue, epilogue0, gather, dstage, autotune, prepare};
    return &t;
  }
};

}  // namespace ld_impl

#define LD_DEFINE_TABLE(P, TT, N) \
  const OpsTable* ops_table_##P##_##N() { return ld_impl::Table<TT, N>::get(); }
