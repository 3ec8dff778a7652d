// ld_irfft_mpi_noalloc: the inverse transform of ld_irfft_mpi for callers that must not allocate
// device memory.  Two kinds of caller need it:
//   * host frameworks that hand out all device memory from their own pool, with a budget fixed
//     at start-up, and forbid driver allocations behind their back, and
//   * time-critical loops that may not allocate after their set-up, because an allocation can
//     synchronise the device, take unbounded time or fail part-way through a run.
// Such a caller cannot create an ld_plan (a plan allocates its twiddle tables and workspace), so
// this entry point keeps its scratch in file-scope device arrays instead: one complex-float buffer
// for an (N, N, N/2+1) spectrum with N <= 64 (64*64*33 complex floats, 1.08 MB) and the twiddle
// tables for N = 16, 32, 64.  Every GPU that loads the library holds these arrays until the process
// exits.  The caller still passes the input and output buffers.
//
// In host code the arrays' names are host-side stand-ins, not device addresses: the first call on
// a device, with that device current, looks their device addresses up with cudaGetSymbolAddress
// and fills the twiddle tables with a synchronous host-to-device copy, and the first call for
// each N launches that size's kernels for the first time (the driver loads them then).  Make the
// first call on each device, and the first call for each N that will be used, before any stream
// capture.
//
// All calls share the one scratch buffer of their device, and each call overwrites it completely
// before reading it.  Calls that overlap on the GPU (different streams, no ordering) race on it.
#include <cmath>
#include <mutex>

#include "ld_ops.cuh"

namespace {

constexpr int NA_NMAX = 64;
constexpr size_t NA_SCRATCH = (size_t)NA_NMAX * NA_NMAX * (NA_NMAX / 2 + 1);
constexpr int NA_MAXDEV = 64;

static __device__ __align__(256) float2 g_na_scratch[NA_SCRATCH];
static __device__ __align__(256) float2 g_na_tw[3][NA_NMAX];  // N = 16, 32, 64

struct NaDevice {
  bool ready = false;
  float2* scratch = nullptr;
  float2* tw = nullptr;
};
NaDevice g_na_dev[NA_MAXDEV];
std::mutex g_na_mutex;

int na_setup(NaDevice** out) {
  int dev = 0;
  LD_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAXDEV) return ld_fail(LD_ERR_UNSUPPORTED, "ld_irfft_mpi_noalloc: device %d", dev);
  std::lock_guard<std::mutex> lock(g_na_mutex);
  NaDevice& d = g_na_dev[dev];
  if (!d.ready) {
    void* s = nullptr;
    void* t = nullptr;
    LD_CUDA_CHECK(cudaGetSymbolAddress(&s, g_na_scratch));
    LD_CUDA_CHECK(cudaGetSymbolAddress(&t, g_na_tw));
    float2 host[3][NA_NMAX];
    for (int i = 0; i < 3; ++i) {
      const int n = 16 << i;
      for (int p = 0; p < NA_NMAX; ++p) {
        const double a = -2.0 * M_PI * (double)(p % n) / (double)n;
        host[i][p] = make_float2((float)std::cos(a), (float)std::sin(a));
      }
    }
    LD_CUDA_CHECK(cudaMemcpy(t, host, sizeof(host), cudaMemcpyHostToDevice));
    d.scratch = (float2*)s;
    d.tw = (float2*)t;
    d.ready = true;
  }
  *out = &d;
  return LD_OK;
}

// x pass (fu -> W), y pass in place on W, z C2R (W -> u): the launch sequence of ld_irfft_mpi
// (Ops::irfft_full) for one component at a time, with W the static scratch.
template <int N>
int na_run(const float2* fu, float* u, int ncomp, float2* W, const float2* tw, cudaStream_t s) {
  using O = ld_impl::Ops<float, N>;
  const int Nf = N / 2 + 1;
  const long long NN = (long long)N * N;
  const long long per = NN * Nf;
  const float sc = (float)(1.0 / ((double)N * N * N));
  for (int c = 0; c < ncomp; ++c) {
    auto xin = O::io(fu + c * per, per, 0, N * Nf, -1);
    auto xout = O::io(W, per, 0, N * Nf, -1);
    // the loaders and storers of Ops::irfft_full (plain rows), so both paths run the same kernels
    if (int rc = O::template colpass<true>(nullptr, KID_XPASS, ld::LdRowsC<float, N, false>{xin},
                                           ld::StRowsC<float, N, false>{xout}, N * Nf, 1, 1, tw, s))
      return rc;
    auto yio = O::io(W, per, (long long)N * Nf, Nf, -1);
    if (int rc = O::template colpass<true>(nullptr, KID_YINV, ld::LdRowsC<float, N, false>{yio},
                                           ld::StRowsC<float, N, false>{yio}, Nf, 1, N, tw, s))
      return rc;
    if (int rc = O::z_c2r(nullptr, W, u + c * NN * N, NN, Nf, Nf, sc, NN * N, per, 1, tw, s)) return rc;
  }
  return LD_OK;
}

}  // namespace

extern "C" int ld_irfft_mpi_noalloc(int n, const void* fu, void* u, int ncomp, void* stream) {
  if (!fu || !u || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_irfft_mpi_noalloc: bad arguments");
  if (n != 16 && n != 32 && n != 64)
    return ld_fail(LD_ERR_UNSUPPORTED,
                   "ld_irfft_mpi_noalloc: N=%d is not supported; the static scratch holds N = 16, 32 or 64 "
                   "(at most 64^3 with 64*64*33 complex floats)", n);
  NaDevice* d = nullptr;
  if (int rc = na_setup(&d)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const float2* tw = d->tw + (n == 16 ? 0 : (n == 32 ? 1 : 2)) * NA_NMAX;
  switch (n) {
    case 16: return na_run<16>((const float2*)fu, (float*)u, ncomp, d->scratch, tw, s);
    case 32: return na_run<32>((const float2*)fu, (float*)u, ncomp, d->scratch, tw, s);
    default: return na_run<64>((const float2*)fu, (float*)u, ncomp, d->scratch, tw, s);
  }
}
