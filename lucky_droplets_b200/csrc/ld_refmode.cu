// The reference's own droplet physics on the GPU (forced-dns-sm.py full_RHS and the RK4 loop,
// F:278-362; particles.py pRHS and the cosine deposition, P:514-577, P:817-837): the number
// density n of small droplets on the grid, advected with the slow-manifold velocity and fed by
// the mass the droplets take up; the droplets (x, v, m) with Stokes drag, settling and growth.
//
// All arithmetic is FP64 (the reference's precision).  Sums are deterministic: clip_zero's
// means come from a fixed partition of the grid reduced in a fixed order, and the deposition is
// a pull over droplets sorted by grid cell that adds, per cell, in the reference's own order
// (stencil offsets a, b, c outermost, droplets by index) with the reference's rounding sequence.
#include <cmath>

#include "ld_internal.cuh"
#include "ld_kernels.cuh"

namespace {

using namespace ld;

constexpr int RED_BLOCKS = 592;  // fixed partition of the reductions (4 per SM)
constexpr int RED_THREADS = 256;

inline int grid1(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

// ---- clip_zero (F:278-285): x <- max(x, 0) * mean(x) / mean(max(x, 0)) ----------------------
__global__ void __launch_bounds__(RED_THREADS)
k_clip_partial(const double* __restrict__ x, long long m, double* __restrict__ part) {
  __shared__ double s0[RED_THREADS], s1[RED_THREADS];
  double a = 0.0, b = 0.0;
  for (long long i = blockIdx.x * (long long)RED_THREADS + threadIdx.x; i < m; i += (long long)RED_BLOCKS * RED_THREADS) {
    const double v = x[i];
    a += v;
    b += v > 0.0 ? v : 0.0;
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  __syncthreads();
  for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}

// part -> [sum x, sum max(x,0)] in fixed order
__global__ void k_clip_final(double* __restrict__ part) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 0.0, b = 0.0;
  for (int i = 0; i < RED_BLOCKS; ++i) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  part[2 * RED_BLOCKS] = a;
  part[2 * RED_BLOCKS + 1] = b;
}

// out = max(src, 0) * oldmean / newmean; with clip_src, src <- max(src, 0) as well (the in-place
// side effect of the reference's clip_zero on its argument)
__global__ void k_clip_apply(double* __restrict__ src, double* __restrict__ out, long long m,
                             const double* __restrict__ sums, int clip_src) {
  const double n3 = (double)m;
  const double oldmean = sums[0] / n3, newmean = sums[1] / n3;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
    const double v = src[i] > 0.0 ? src[i] : 0.0;
    if (clip_src) src[i] = v;
    out[i] = __ddiv_rn(__dmul_rn(v, oldmean), newmean);
  }
}

// ---- RK4 bookkeeping ------------------------------------------------------------------------
// y += a x
__global__ void k_axpy(double* __restrict__ y, double a, const double* __restrict__ x, long long m) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    y[i] = __dadd_rn(y[i], __dmul_rn(a, x[i]));
}
// z = x + a y
__global__ void k_waxpy(double* __restrict__ z, const double* __restrict__ x, double a, const double* __restrict__ y,
                        long long m) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    z[i] = __dadd_rn(x[i], __dmul_rn(y[i], a));
}

// ---- n field (F:325-330) ---------------------------------------------------------------------
// nv_c = n * v_c (planar 3 x m)
__global__ void k_nv(const double* __restrict__ n, const double* __restrict__ v, double* __restrict__ nv, long long m) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
    const double a = n[i];
    nv[i] = a * v[i];
    nv[m + i] = a * v[m + i];
    nv[2 * m + i] = a * v[2 * m + i];
  }
}

// knk = -i (kx nvk_x + ky nvk_y + kz nvk_z) - fck on the cube
__global__ void k_n_combine(const double2* __restrict__ nvk, const double2* __restrict__ fck, double2* __restrict__ knk,
                            long long cs, int kc, int My, int Mzp) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cs; e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / ((long long)My * Mzp)), iy = (int)((e / Mzp) % My), kz = (int)(e % Mzp);
    const double kx = ix <= kc ? ix : ix - My, ky = iy <= kc ? iy : iy - My;
    const double2 a = nvk[e], b = nvk[cs + e], c = nvk[2 * cs + e], f = fck[e];
    const double re = kx * a.x + ky * b.x + kz * c.x, im = kx * a.y + ky * b.y + kz * c.y;
    knk[e] = make_double2(im - f.x, -re - f.y);  // -i (re + i im) = im - i re
  }
}

// ---- droplets (P:817-837) ---------------------------------------------------------------------
struct RefDrop {
  double factor, growthfactor, st_s, tau_eta, g;
};

// coord (n, 7): x, v, m; iu, iv (n, 3) fluid and slow-manifold velocity at the droplets, ic (n)
// the number density there -> kp (n, 7), mdot (n)
__global__ void k_prhs_ref(const double* __restrict__ coord, const double* __restrict__ iu, const double* __restrict__ iv,
                           const double* __restrict__ ic, long long n, RefDrop P, double* __restrict__ kp,
                           double* __restrict__ mdot) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double* c = coord + 7 * i;
    const double st = pow(c[6] / P.factor, 2.0 / 3.0);                               // P:823
    const double d0 = c[3] - iv[3 * i], d1 = c[4] - iv[3 * i + 1], d2 = c[5] - iv[3 * i + 2];
    const double rel = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    const double q = 1.0 + sqrt(P.st_s / st);
    const double md = P.growthfactor * (q * q) * ic[i] * rel;                          // P:828
    double* k = kp + 7 * i;
    k[0] = c[3];
    k[1] = c[4];
    k[2] = c[5];                                                                      // P:831
    const double den = st * P.tau_eta;
    k[3] = (iu[3 * i] - c[3]) / den;
    k[4] = (iu[3 * i + 1] - c[4]) / den;
    k[5] = (iu[3 * i + 2] - c[5]) / den - P.g;                                        // P:832, P:834
    k[6] = md;                                                                        // P:835
    mdot[i] = md;
  }
}

// Grid cell (P:441: idx = pos // dx of the wrapped position) and cosine weights of every droplet:
// key = (ix N + iy) N + iz, w (n, 12): the four weights along x, y, z (P:9-16, P:454-456).
__global__ void k_cell_weights(const double* __restrict__ coord, long long n, int N, double L,
                               unsigned* __restrict__ key, unsigned* __restrict__ val, double* __restrict__ w) {
  const double dx = L / double(N);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int idx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double p = coord[7 * i + a] - L * floor(coord[7 * i + a] / L);
      long long ii = (long long)floor(p / dx);
      idx[a] = (int)(((ii % N) + N) % N);
      // X_j at the periodic index j = (idx + o) mod N, o = -1..2
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        const long long j = (((ii + o - 1) % N) + N) % N;
        const double X = dx * (double)j;
        w[12 * i + 4 * a + o] = (1.0 + cos((p - X) * (M_PI / (2.0 * dx)))) / 4.0;
      }
    }
    key[i] = (unsigned)(((long long)idx[0] * N + idx[1]) * N + idx[2]);
    val[i] = (unsigned)i;
  }
}

// cs[k] = number of sorted keys < k, k = 0..ncell
__global__ void k_starts(const unsigned* __restrict__ skey, long long n, long long ncell, int* __restrict__ cs) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k <= ncell; k += (long long)gridDim.x * blockDim.x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if ((long long)skey[mid] < k) lo = mid + 1;
      else hi = mid;
    }
    cs[k] = (int)lo;
  }
}

// fc[j] = sum over stencil offsets (a, b, c) and droplets p (by index) whose stencil covers j of
// mdot_p wx_p[a] wy_p[b] wz_p[c] / dx^3, added in the reference's order (P:560-577).
__global__ void k_deposit_pull(const unsigned* __restrict__ sval, const int* __restrict__ cs,
                               const double* __restrict__ w, const double* __restrict__ mdot, int N, double dx3,
                               double* __restrict__ fc) {
  const long long m = (long long)N * N * N;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x) {
    const int jx = (int)(e / ((long long)N * N)), jy = (int)((e / N) % N), jz = (int)(e % N);
    double acc = 0.0;
    for (int a = 0; a < 4; ++a) {
      const int ix = (jx + 1 - a + N) % N;  // a droplet in cell i covers i - 1 + a
      for (int b = 0; b < 4; ++b) {
        const int iy = (jy + 1 - b + N) % N;
        for (int c = 0; c < 4; ++c) {
          const int iz = (jz + 1 - c + N) % N;
          const long long cell = ((long long)ix * N + iy) * N + iz;
          for (int t = cs[cell]; t < cs[cell + 1]; ++t) {
            const unsigned p = sval[t];
            const double* wp = w + 12 * (long long)p;
            const double v = __dmul_rn(__dmul_rn(__dmul_rn(mdot[p], wp[a]), wp[4 + b]), wp[8 + c]);
            acc = __dadd_rn(acc, __ddiv_rn(v, dx3));
          }
        }
      }
    }
    fc[e] = acc;
  }
}

// pos (n, 3) = coord[:, 0:3]
__global__ void k_extract_pos(const double* __restrict__ coord, long long n, double* __restrict__ pos) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 3 * n; e += (long long)gridDim.x * blockDim.x)
    pos[e] = coord[7 * (e / 3) + e % 3];
}

}  // namespace

extern "C" {

int ld_extract_pos(const double* coord, int64_t n, double* pos, void* stream) {
  if (n < 0 || (n > 0 && (!coord || !pos))) return ld_fail(LD_ERR_ARG, "ld_extract_pos: bad arguments");
  if (n == 0) return LD_OK;
  k_extract_pos<<<grid1(3 * n), 256, 0, (cudaStream_t)stream>>>(coord, n, pos);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int64_t ld_ref_workspace_doubles() { return 2 * RED_BLOCKS + 2; }

int ld_clip_zero(double* x, double* out, int64_t m, int clip_src, double* work, void* stream) {
  if (!x || !out || !work || m < 1) return ld_fail(LD_ERR_ARG, "ld_clip_zero: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  k_clip_partial<<<RED_BLOCKS, RED_THREADS, 0, s>>>(x, m, work);
  k_clip_final<<<1, 32, 0, s>>>(work);
  k_clip_apply<<<grid1(m), 256, 0, s>>>(x, out, m, work + 2 * RED_BLOCKS, clip_src);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_axpy(double* y, double a, const double* x, int64_t m, void* stream) {
  if (m < 0 || (m > 0 && (!y || !x))) return ld_fail(LD_ERR_ARG, "ld_axpy: bad arguments");
  if (m == 0) return LD_OK;
  k_axpy<<<grid1(m), 256, 0, (cudaStream_t)stream>>>(y, a, x, m);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_waxpy(double* z, const double* x, double a, const double* y, int64_t m, void* stream) {
  if (m < 0 || (m > 0 && (!z || !x || !y))) return ld_fail(LD_ERR_ARG, "ld_waxpy: bad arguments");
  if (m == 0) return LD_OK;
  k_waxpy<<<grid1(m), 256, 0, (cudaStream_t)stream>>>(z, x, a, y, m);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_n_products(ld_plan* p, const double* n, const double* v, double* nv, void* stream) {
  if (!p || p->prec != LD_F64 || !n || !v || !nv) return ld_fail(LD_ERR_ARG, "ld_n_products: bad arguments (FP64 plans)");
  const long long m = (long long)p->N * p->N * p->N;
  k_nv<<<grid1(m), 256, 0, (cudaStream_t)stream>>>(n, v, nv, m);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_n_combine(ld_plan* p, const void* nvk, const void* fck, void* knk, void* stream) {
  if (!p || p->prec != LD_F64 || !nvk || !fck || !knk) return ld_fail(LD_ERR_ARG, "ld_n_combine: bad arguments (FP64 plans)");
  const long long cs = p->cube_elems();
  k_n_combine<<<grid1(cs), 256, 0, (cudaStream_t)stream>>>((const double2*)nvk, (const double2*)fck, (double2*)knk,
                                                            cs, p->kc, p->My, p->Mzp);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_prhs_ref(const double* coord, const double* iu, const double* iv, const double* ic, int64_t n, double factor,
                double growthfactor, double st_s, double tau_eta, double g, double* kp, double* mdot, void* stream) {
  if (n < 0 || (n > 0 && (!coord || !iu || !iv || !ic || !kp || !mdot))) return ld_fail(LD_ERR_ARG, "ld_prhs_ref: bad arguments");
  if (n == 0) return LD_OK;
  RefDrop P{factor, growthfactor, st_s, tau_eta, g};
  k_prhs_ref<<<grid1(n), 256, 0, (cudaStream_t)stream>>>(coord, iu, iv, ic, n, P, kp, mdot);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_cell_weights(const double* coord, int64_t n, int N, double L, uint32_t* key, uint32_t* val, double* w,
                    void* stream) {
  if (n < 0 || N < 4 || (n > 0 && (!coord || !key || !val || !w))) return ld_fail(LD_ERR_ARG, "ld_cell_weights: bad arguments");
  if (n == 0) return LD_OK;
  k_cell_weights<<<grid1(n), 256, 0, (cudaStream_t)stream>>>(coord, n, N, L, key, val, w);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_cell_starts(const uint32_t* skey, int64_t n, int64_t ncell, int32_t* cs, void* stream) {
  if (n < 0 || ncell < 1 || !cs || (n > 0 && !skey)) return ld_fail(LD_ERR_ARG, "ld_cell_starts: bad arguments");
  k_starts<<<grid1(ncell + 1), 256, 0, (cudaStream_t)stream>>>(skey, n, ncell, cs);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_deposit_pull(const uint32_t* sval, const int32_t* cs, const double* w, const double* mdot, int N, double L,
                    double* fc, void* stream) {
  if (N < 4 || !cs || !fc) return ld_fail(LD_ERR_ARG, "ld_deposit_pull: bad arguments");
  const double dx = L / double(N);
  const double dx3 = pow(dx, 3.0);
  const long long m = (long long)N * N * N;
  k_deposit_pull<<<grid1(m), 256, 0, (cudaStream_t)stream>>>(sval, cs, w, mdot, N, dx3, fc);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

}  // extern "C"
