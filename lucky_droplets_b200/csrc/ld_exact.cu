// Exact spectral (direct Fourier sum) velocity at arbitrary points, FP64.
//
//   u_c(x) = (1/N^3) sum_{kx,ky} sum_{kz=0}^{kc} w_kz Re( uk_c(kx,ky,kz) exp(i k.x) ),
//   w_0 = 1, w_kz = 2 (kz > 0),
// the continuous extension of the inverse real transform (at grid points it equals irfft, which
// also drops the imaginary part of the kz = 0 coefficients).  Only the modes of the spherical
// mask round(|k|) <= kc are summed: they are the only non-zero modes of a dealiased field.
//
// One thread per point.  Every thread of a warp walks the same (kx, ky, kz) sequence, so the
// spectrum loads are warp-uniform (one broadcast transaction per warp); the phases come from
// FP64 recurrences seeded by sincos once per row.
#include "ld_internal.cuh"

namespace {

template <typename T>
__global__ void __launch_bounds__(128)
k_exact_sum(const ld::cplx<T>* __restrict__ uk, long long cs, int N, int kc, int My, int Mzp,
            const double* __restrict__ pos, long long n, double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool ok = i < n;
  const double x = ok ? pos[3 * i] : 0.0, y = ok ? pos[3 * i + 1] : 0.0, z = ok ? pos[3 * i + 2] : 0.0;
  const int lim = kc * kc + kc;  // round(|k|) <= kc  <=>  k^2 <= kc^2 + kc
  double sxr, sxi, syr, syi, szr, szi;
  sincos(x, &sxi, &sxr);  // exp(i x)
  sincos(y, &syi, &syr);
  sincos(z, &szi, &szr);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int ix = 0; ix < My; ++ix) {
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
        double ty[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        double ezr = 1.0, ezi = 0.0;
        for (int kz = 0; kz <= kc && r2 + kz * kz <= lim; ++kz) {
          const double w = kz ? 2.0 : 1.0;
          const double wr = w * ezr, wi = w * ezi;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const ld::cplx<T> v = uk[c * cs + base + kz];
            const double vr = (double)v.x, vi = (double)v.y;
            ty[c][0] += vr * wr - vi * wi;
            ty[c][1] += vr * wi + vi * wr;
          }
          const double t = ezr * szr - ezi * szi;
          ezi = ezr * szi + ezi * szr;
          ezr = t;
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
  if (ok) {
    const double s = 1.0 / ((double)N * N * N);
    for (int c = 0; c < 3; ++c) out[3 * i + c] = acc[c] * s;
  }
}

}  // namespace

extern "C" int ld_exact_sum(ld_plan* p, const void* uk, const double* pos, int64_t n, double* out, void* stream) {
  if (!p || !uk || !pos || !out || n < 0) return ld_fail(LD_ERR_ARG, "ld_exact_sum: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  ProfScope ps(p, KID_EXACT, s);
  const int th = 128;
  const long long blocks = (n + th - 1) / th;
  if (p->prec == LD_F32)
    k_exact_sum<float><<<(unsigned)blocks, th, 0, s>>>((const float2*)uk, p->cube_elems(), p->N, p->kc, p->My,
                                                       p->Mzp, pos, n, out);
  else
    k_exact_sum<double><<<(unsigned)blocks, th, 0, s>>>((const double2*)uk, p->cube_elems(), p->N, p->kc, p->My,
                                                        p->Mzp, pos, n, out);
  LD_LAUNCH_CHECK();
  return LD_OK;
}
