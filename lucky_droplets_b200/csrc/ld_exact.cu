// Exact spectral (direct Fourier sum) velocity at arbitrary points, FP64.
//
//   u_c(x) = (1/N^3) sum_{kx,ky} sum_{kz=0}^{kc} w_kz Re( uk_c(kx,ky,kz) exp(i k.x) ),
//   w_0 = 1, w_kz = 2 (kz > 0),
// the continuous extension of the inverse real transform (at grid points it equals irfft, which
// also drops the imaginary part of the kz = 0 coefficients).  Only the modes of the spherical
// mask round(|k|) <= kc are summed: they are the only non-zero modes of a dealiased field.
//
// Thread per point and block per (tile of 128 points, chunk of kx planes): the kx planes are
// split across blocks so that even 1e4 points fill the GPU, and the per-chunk partial sums are
// added in chunk order afterwards (deterministic).  Every thread of a warp walks the same
// (kx, ky, kz) sequence, so the spectrum loads are warp-uniform (one broadcast transaction per
// warp); the phases come from FP64 recurrences seeded by sincos once per row.  Along kz the
// weight-2 terms accumulate unweighted in fused multiply-adds and are doubled once per row.
#include "ld_internal.cuh"

namespace {

template <typename T>
__global__ void __launch_bounds__(128)
k_exact_sum(const ld::cplx<T>* __restrict__ uk, long long cs, int N, int kc, int My, int Mzp,
            const double* __restrict__ pos, long long n, int per_chunk, double* __restrict__ part) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int ix0 = blockIdx.y * per_chunk;
  const int ix1 = ix0 + per_chunk < My ? ix0 + per_chunk : My;
  const bool ok = i < n;
  const double x = ok ? pos[3 * i] : 0.0, y = ok ? pos[3 * i + 1] : 0.0, z = ok ? pos[3 * i + 2] : 0.0;
  const int lim = kc * kc + kc;  // round(|k|) <= kc  <=>  k^2 <= kc^2 + kc
  double sxr, sxi, syr, syi, szr, szi;
  sincos(x, &sxi, &sxr);  // exp(i x)
  sincos(y, &syi, &syr);
  sincos(z, &szi, &szr);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int ix = ix0; ix < ix1; ++ix) {
    const int kx = ix <= kc ? ix : ix - My;
    double exr, exi;
    sincos((double)kx * x, &exi, &exr);
    double tx[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    // ky runs 0..kc, then -kc..-1: restart the recurrence at -kc
    double eyr = 1.0, eyi = 0.0;
    for (int iy = 0; iy < My; ++iy) {
      const int ky = iy <= kc ? iy : iy - My;
      if (iy == kc + 1) sincos(-(double)kc * y, &eyi, &eyr);
      const int r2 = kx * kx + ky * ky;
      if (r2 <= lim) {
        const long long base = ((long long)ix * My + iy) * Mzp;
        // kz = 0 (weight 1) seeds the sum; the kz > 0 terms (weight 2) accumulate in fused
        // multiply-adds and are doubled once at the end of the row
        double t0[3][2], ty[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const ld::cplx<T> v = uk[c * cs + base];
          t0[c][0] = (double)v.x;
          t0[c][1] = (double)v.y;
        }
        double ezr = szr, ezi = szi;
        for (int kz = 1; kz <= kc && r2 + kz * kz <= lim; ++kz) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const ld::cplx<T> v = uk[c * cs + base + kz];
            const double vr = (double)v.x, vi = (double)v.y;
            ty[c][0] = fma(vr, ezr, fma(-vi, ezi, ty[c][0]));
            ty[c][1] = fma(vr, ezi, fma(vi, ezr, ty[c][1]));
          }
          const double t = fma(ezr, szr, -ezi * szi);
          ezi = fma(ezr, szi, ezi * szr);
          ezr = t;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ty[c][0] = fma(2.0, ty[c][0], t0[c][0]);
          ty[c][1] = fma(2.0, ty[c][1], t0[c][1]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          tx[c][0] += ty[c][0] * eyr - ty[c][1] * eyi;
          tx[c][1] += ty[c][0] * eyi + ty[c][1] * eyr;
        }
      }
      const double t = eyr * syr - eyi * syi;
      eyi = eyr * syi + eyi * syr;
      eyr = t;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += tx[c][0] * exr - tx[c][1] * exi;  // Re(ex * tx)
  }
  if (ok)
    for (int c = 0; c < 3; ++c) part[((long long)blockIdx.y * n + i) * 3 + c] = acc[c];
}

// out = (1/N^3) sum over chunks, in chunk order
__global__ void k_exact_reduce(const double* __restrict__ part, int chunks, long long n, double scale,
                               double* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 3 * n; e += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < chunks; ++c) s += part[(long long)c * 3 * n + e];
    out[e] = s * scale;
  }
}

// FP32 spectrum -> FP64 copy (exact), so that the sum converts nothing per mode.
__global__ void k_spec_to_f64(const float2* __restrict__ in, double2* __restrict__ out, long long m) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x) {
    const float2 v = in[e];
    out[e] = make_double2((double)v.x, (double)v.y);
  }
}

}  // namespace

extern "C" int ld_exact_sum(ld_plan* p, const void* uk, const double* pos, int64_t n, double* out, void* stream) {
  if (!p || !uk || !pos || !out || n < 0) return ld_fail(LD_ERR_ARG, "ld_exact_sum: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  ProfScope ps(p, KID_EXACT, s);
  const int th = 128;
  // partial sums live in the plan's transform workspace (free between steps): points are taken
  // in batches that fit it
  long long cap = (long long)(p->work_bytes / sizeof(double));
  double* part = (double*)p->work;
  // FP32 plans: an FP64 copy of the spectrum at the end of the workspace when it leaves room for
  // the partial sums of one batch of points (the sum then converts nothing per mode)
  const double2* uk64 = nullptr;
  if (p->prec == LD_F32) {
    const long long m = 3 * p->cube_elems();
    const size_t copy_bytes = ((size_t)m * sizeof(double2) + 255) / 256 * 256;
    const long long rest = (long long)((p->work_bytes - (copy_bytes < p->work_bytes ? copy_bytes : p->work_bytes)) /
                                       sizeof(double));
    if (copy_bytes < p->work_bytes && rest >= 3LL * p->My * (n < 4096 ? n : 4096)) {
      double2* dst = (double2*)((char*)p->work + (p->work_bytes - copy_bytes) / 256 * 256);
      long long gb = (m + 255) / 256;
      if (gb > 148LL * 16) gb = 148LL * 16;
      k_spec_to_f64<<<(unsigned)gb, 256, 0, s>>>((const float2*)uk, dst, m);
      uk64 = dst;
      cap = (long long)(((char*)dst - (char*)p->work) / sizeof(double));
    }
  }
  const double scale = 1.0 / ((double)p->N * p->N * p->N);
  for (long long b0 = 0; b0 < n; ) {
    long long nb = n - b0;
    const long long tiles_all = (nb + th - 1) / th;
    int chunks = (int)((148LL * 12 + tiles_all - 1) / tiles_all);
    if (chunks > p->My) chunks = p->My;
    if (chunks < 1) chunks = 1;
    if ((long long)chunks * 3 * nb > cap) {
      nb = cap / (3LL * chunks);
      if (nb < 1) { chunks = 1; nb = cap / 3; }
      if (nb < 1) return ld_fail(LD_ERR_CAPACITY, "ld_exact_sum: no workspace");
    }
    const int per_chunk = (p->My + chunks - 1) / chunks;
    chunks = (p->My + per_chunk - 1) / per_chunk;
    const dim3 grid((unsigned)((nb + th - 1) / th), (unsigned)chunks);
    if (uk64)
      k_exact_sum<double><<<grid, th, 0, s>>>(uk64, p->cube_elems(), p->N, p->kc, p->My, p->Mzp, pos + 3 * b0, nb,
                                              per_chunk, part);
    else if (p->prec == LD_F32)
      k_exact_sum<float><<<grid, th, 0, s>>>((const float2*)uk, p->cube_elems(), p->N, p->kc, p->My, p->Mzp,
                                             pos + 3 * b0, nb, per_chunk, part);
    else
      k_exact_sum<double><<<grid, th, 0, s>>>((const double2*)uk, p->cube_elems(), p->N, p->kc, p->My, p->Mzp,
                                              pos + 3 * b0, nb, per_chunk, part);
    long long rb = (3 * nb + 255) / 256;
    if (rb > 148LL * 16) rb = 148LL * 16;
    k_exact_reduce<<<(unsigned)rb, 256, 0, s>>>(part, chunks, nb, scale, out + 3 * b0);
    LD_LAUNCH_CHECK();
    b0 += nb;
  }
  return LD_OK;
}
