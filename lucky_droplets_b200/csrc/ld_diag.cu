// Diagnostics of the reference's output step (F:419-484): the cross spectrum behind the flux
// spectrum Pi(k) (F:425-428) and the spectral divergence (F:216-230, printed at F:472); and the
// region copies between the reference's spectral layout and the dealiased cube.
#include <cmath>

#include "ld_internal.cuh"
#include "ld_kernels.cuh"

namespace {

using namespace ld;

// Per shell s (one CTA, fixed-order FP64 reduction): sum over its modes of
// Re(conj(a) . b) * w * norm0 with the Hermitian weight w of F:136.
template <typename T>
__global__ void k_shell_cross(const cplx<T>* __restrict__ a, const cplx<T>* __restrict__ b, long long cs,
                              const int* __restrict__ off, const int* __restrict__ idx, int Mzp, double norm0,
                              double* __restrict__ out) {
  __shared__ double red[256];
  const int s = blockIdx.x;
  double acc = 0.0;
  for (int t = off[s] + threadIdx.x; t < off[s + 1]; t += blockDim.x) {
    const int e = idx[t];
    const double w = (e % Mzp) ? 2.0 : 1.0;
    double m = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cplx<T> x = a[c * cs + e], y = b[c * cs + e];
      m += double(x.x) * double(y.x) + double(x.y) * double(y.y);
    }
    acc += m * w * norm0;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[s] = red[0];
}

// div_hat = i (kx u + ky v + kz w) on the cube (one component out).
template <typename T>
__global__ void k_div_spec(const cplx<T>* __restrict__ u, cplx<T>* __restrict__ out, long long cs, int kc, int My,
                           int Mzp) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cs; e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / ((long long)My * Mzp)), iy = (int)((e / Mzp) % My), kz = (int)(e % Mzp);
    const T kx = T(ix <= kc ? ix : ix - My), ky = T(iy <= kc ? iy : iy - My);
    const cplx<T> a = u[e], b = u[cs + e], c = u[2 * cs + e];
    const T re = kx * a.x + ky * b.x + T(kz) * c.x, im = kx * a.y + ky * b.y + T(kz) * c.y;
    out[e] = cmk(-im, re);
  }
}

// Zero every cube mode outside the spherical mask round(|k|) <= kc (F:129), kz padding included.
template <typename T>
__global__ void k_cube_mask(cplx<T>* __restrict__ u, long long total, int kc, int My, int Mzp) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / Mzp;
    const int kz = (int)(e - r * Mzp);
    const int iy = (int)(r % My), ix = (int)((r / My) % My);
    const int kx = ix <= kc ? ix : ix - My, ky = iy <= kc ? iy : iy - My;
    if (kz > kc || kx * kx + ky * ky + kz * kz > kc * kc + kc) u[e] = czero<cplx<T>>();
  }
}

inline int grid1(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" {

int ld_shell_cross(ld_plan* p, const void* a, const void* b, double* out, void* stream) {
  if (!p || !a || !b || !out) return ld_fail(LD_ERR_ARG, "ld_shell_cross: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const double norm0 = std::pow(2.0 * M_PI, 3) / std::pow((double)p->N, 6);
  if (p->prec == LD_F32)
    k_shell_cross<float><<<p->Nf, 256, 0, s>>>((const float2*)a, (const float2*)b, p->cube_elems(), p->shell_off,
                                               p->shell_idx, p->Mzp, norm0, out);
  else
    k_shell_cross<double><<<p->Nf, 256, 0, s>>>((const double2*)a, (const double2*)b, p->cube_elems(),
                                                p->shell_off, p->shell_idx, p->Mzp, norm0, out);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_divergence_spec(ld_plan* p, const void* uk, void* divk, void* stream) {
  if (!p || !uk || !divk) return ld_fail(LD_ERR_ARG, "ld_divergence_spec: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const long long cs = p->cube_elems();
  if (p->prec == LD_F32)
    k_div_spec<float><<<grid1(cs), 256, 0, s>>>((const float2*)uk, (float2*)divk, cs, p->kc, p->My, p->Mzp);
  else
    k_div_spec<double><<<grid1(cs), 256, 0, s>>>((const double2*)uk, (double2*)divk, cs, p->kc, p->My, p->Mzp);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_spec_copy_region(ld_plan* p, const void* src, void* dst, int ncomp, int direction, void* stream) {
  if (!p || !src || !dst || ncomp < 1 || (direction != 0 && direction != 1))
    return ld_fail(LD_ERR_ARG, "ld_spec_copy_region: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int N = p->N, kc = p->kc, My = p->My, Mzp = p->Mzp, Nf = p->Nf;
  const size_t ce = 2 * p->esz;  // bytes per complex element
  // the four (kx, ky) blocks of the cube: frequencies 0..kc and -kc..-1 along each axis
  const int full0[2] = {0, N - kc}, cube0[2] = {0, kc + 1}, cnt[2] = {kc + 1, kc};
  void* fullp = const_cast<void*>(direction == 0 ? src : dst);
  void* cubep = const_cast<void*>(direction == 0 ? dst : src);
  cudaPitchedPtr fpp = make_cudaPitchedPtr(fullp, (size_t)Nf * ce, (size_t)Nf * ce, (size_t)N);
  cudaPitchedPtr cpp = make_cudaPitchedPtr(cubep, (size_t)Mzp * ce, (size_t)Mzp * ce, (size_t)My);
  for (int c = 0; c < ncomp; ++c)
    for (int bx = 0; bx < 2; ++bx)
      for (int by = 0; by < 2; ++by) {
        if (cnt[bx] == 0 || cnt[by] == 0) continue;
        cudaMemcpy3DParms m = {};
        const cudaPos fpos = make_cudaPos(0, (size_t)full0[by], (size_t)c * N + full0[bx]);
        const cudaPos cpos = make_cudaPos(0, (size_t)cube0[by], (size_t)c * My + cube0[bx]);
        if (direction == 0) { m.srcPtr = fpp; m.srcPos = fpos; m.dstPtr = cpp; m.dstPos = cpos; }
        else { m.srcPtr = cpp; m.srcPos = cpos; m.dstPtr = fpp; m.dstPos = fpos; }
        m.extent = make_cudaExtent((size_t)(kc + 1) * ce, (size_t)cnt[by], (size_t)cnt[bx]);
        m.kind = cudaMemcpyDefault;
        LD_CUDA_CHECK(cudaMemcpy3DAsync(&m, s));
      }
  if (direction == 0) {
    const long long total = p->cube_elems() * ncomp;
    if (p->prec == LD_F32) k_cube_mask<float><<<grid1(total), 256, 0, s>>>((float2*)cubep, total, kc, My, Mzp);
    else k_cube_mask<double><<<grid1(total), 256, 0, s>>>((double2*)cubep, total, kc, My, Mzp);
    LD_LAUNCH_CHECK();
  }
  return LD_OK;
}

}  // extern "C"
