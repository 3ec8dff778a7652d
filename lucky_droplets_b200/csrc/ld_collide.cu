// Cell-list collision detection and the stable LSD radix sort it uses.
//
// Pipeline (one call of ld_collide):
//   keys      key[i] = cell of the wrapped position of droplet i, val[i] = i
//   sort      stable LSD radix sort of (key, val), 8-bit digits
//   ranges    cell_start / cell_end of every cell in the sorted order
//   reorder   sorted copies of wrapped positions and radii (candidate loads become contiguous)
//   count     per droplet i: partners j > i among the 27 neighbour cells that overlap
//   scan      exclusive scan of the counts in droplet-id order -> offsets, total
//   emit      pairs (i, j) at offset[i] + t, each droplet's run sorted by j
// The FP64 arithmetic (wrap, cell index, minimum image, squared distance) is done with explicit
// round-to-nearest operations and no fused multiply-add, in the same order as the CPU rule, so
// the pair list is bit-exact given identical inputs.
#include <cstdio>
#include <new>

#include "ld_internal.cuh"

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RADIX = 256;

__device__ __forceinline__ double wrapL(double x, double L) {
  return __dsub_rn(x, __dmul_rn(L, floor(__ddiv_rn(x, L))));
}

__device__ __forceinline__ int cell_of(double p, double cw, int nc) {
  int c = (int)__ddiv_rn(p, cw);
  return c < nc - 1 ? c : nc - 1;
}

__global__ void k_cell_keys(const double* __restrict__ pos, long long n, double L, double cw, int nc,
                            unsigned* __restrict__ key, unsigned* __restrict__ val) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cx = cell_of(wrapL(pos[3 * i], L), cw, nc);
    const int cy = cell_of(wrapL(pos[3 * i + 1], L), cw, nc);
    const int cz = cell_of(wrapL(pos[3 * i + 2], L), cw, nc);
    key[i] = (unsigned)((cx * nc + cy) * nc + cz);
    val[i] = (unsigned)i;
  }
}

// ---- radix sort -------------------------------------------------------------------------------
__global__ void __launch_bounds__(RS_THREADS)
k_rs_hist(const unsigned* __restrict__ key, long long n, int shift, unsigned* __restrict__ hist, int nblocks) {
  __shared__ unsigned cnt[RADIX];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * RS_TILE;
  for (int r = 0; r < RS_ITEMS; ++r) {
    const long long i = base + r * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(key[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * (long long)nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// Exclusive scan in place of m unsigned counts, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_u32(unsigned* __restrict__ a, long long m) {
  __shared__ unsigned part[1024];
  const int t = threadIdx.x;
  const long long per = (m + 1023) / 1024;
  const long long lo = t * per, hi = lo + per < m ? lo + per : m;
  unsigned s = 0;
  for (long long i = lo; i < hi; ++i) s += a[i];
  part[t] = s;
  __syncthreads();
  for (int w = 1; w < 1024; w <<= 1) {
    unsigned v = t >= w ? part[t - w] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  unsigned run = t ? part[t - 1] : 0;
  for (long long i = lo; i < hi; ++i) {
    const unsigned v = a[i];
    a[i] = run;
    run += v;
  }
}

// Stable scatter: items are ranked in index order within the tile (round by round, warp by warp).
__global__ void __launch_bounds__(RS_THREADS)
k_rs_scatter(const unsigned* __restrict__ kin, const unsigned* __restrict__ vin, unsigned* __restrict__ kout,
             unsigned* __restrict__ vout, long long n, int shift, const unsigned* __restrict__ off, int nblocks) {
  constexpr int W = RS_THREADS / 32;
  __shared__ unsigned base[RADIX];
  __shared__ unsigned wcnt[W][RADIX];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  base[t] = off[t * (long long)nblocks + blockIdx.x];
  const long long tile = (long long)blockIdx.x * RS_TILE;
  const unsigned lt = (1u << lane) - 1u;
  for (int r = 0; r < RS_ITEMS; ++r) {
    for (int d = t; d < W * RADIX; d += RS_THREADS) (&wcnt[0][0])[d] = 0;
    __syncthreads();
    const long long i = tile + r * RS_THREADS + t;
    const bool ok = i < n;
    const unsigned k = ok ? kin[i] : 0u;
    const unsigned v = ok ? vin[i] : 0u;
    const int dig = ok ? (int)((k >> shift) & 0xff) : RADIX;  // RADIX: no item
    const unsigned peers = __match_any_sync(0xffffffffu, dig);
    const unsigned rank_w = __popc(peers & lt);
    if (ok && rank_w == 0) wcnt[w][dig] = __popc(peers);
    __syncthreads();
    if (ok) {
      unsigned before = 0;
      for (int q = 0; q < w; ++q) before += wcnt[q][dig];
      const unsigned dst = base[dig] + before + rank_w;
      kout[dst] = k;
      vout[dst] = v;
    }
    __syncthreads();
    unsigned tot = 0;
    for (int q = 0; q < W; ++q) tot += wcnt[q][t];
    base[t] += tot;
    __syncthreads();
  }
}

// ---- cell ranges and sorted copies ------------------------------------------------------------
__global__ void k_cell_ranges(const unsigned* __restrict__ skey, long long n, int* __restrict__ start,
                              int* __restrict__ end) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const unsigned k = skey[s];
    if (s == 0 || skey[s - 1] != k) start[k] = (int)s;
    if (s == n - 1 || skey[s + 1] != k) end[k] = (int)(s + 1);
  }
}

__global__ void k_sorted_copy(const double* __restrict__ pos, const double* __restrict__ rad,
                              const unsigned* __restrict__ sval, long long n, double L, double4* __restrict__ sp) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const unsigned i = sval[s];
    double4 q;
    q.x = wrapL(pos[3 * (long long)i], L);
    q.y = wrapL(pos[3 * (long long)i + 1], L);
    q.z = wrapL(pos[3 * (long long)i + 2], L);
    q.w = rad[i];
    sp[s] = q;
  }
}

__device__ __forceinline__ double min_image(double d, double L) {
  const double h = 0.5 * L;
  if (d > h) d = __dsub_rn(d, L);
  if (d < -h) d = __dadd_rn(d, L);
  return d;
}

__device__ __forceinline__ bool overlap(const double4 a, const double4 b, double L) {
  const double dx = min_image(__dsub_rn(a.x, b.x), L);
  const double dy = min_image(__dsub_rn(a.y, b.y), L);
  const double dz = min_image(__dsub_rn(a.z, b.z), L);
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  const double rs = __dadd_rn(a.w, b.w);
  return d2 < __dmul_rn(rs, rs);
}

// MODE 0: count partners per droplet id; MODE 1: emit pairs.
template <int MODE>
__global__ void k_pairs(const double4* __restrict__ sp, const unsigned* __restrict__ sval,
                        const unsigned* __restrict__ skey, const int* __restrict__ start, const int* __restrict__ end,
                        long long n, int nc, double L, unsigned* __restrict__ cnt, const unsigned* __restrict__ off,
                        int* __restrict__ pairs, long long cap) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const double4 me = sp[s];
    const unsigned id = sval[s];
    const int key = (int)skey[s];
    const int cz = key % nc, cy = (key / nc) % nc, cx = key / (nc * nc);
    unsigned c = 0;
    long long o = 0, o_end = 0;
    if (MODE == 1) { o = off[id]; o_end = o + (off[id + 1] - off[id]); }
    // neighbour cells; with nc < 3 a cell can repeat, so distinct cells only
    int seen[27];
    int ns = 0;
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b)
        for (int d = -1; d <= 1; ++d) {
          const int nx = (cx + a + nc) % nc, ny = (cy + b + nc) % nc, nz = (cz + d + nc) % nc;
          const int nk = (nx * nc + ny) * nc + nz;
          bool dup = false;
          for (int q = 0; q < ns; ++q) dup |= seen[q] == nk;
          if (dup) continue;
          seen[ns++] = nk;
          const int e = end[nk];
          for (int t = start[nk]; t < e; ++t) {
            const unsigned jd = sval[t];
            if (jd <= id) continue;
            if (overlap(me, sp[t], L)) {
              if (MODE == 0) ++c;
              else {
                if (o < cap) { pairs[2 * o] = (int)id; pairs[2 * o + 1] = (int)jd; }
                ++o;
              }
            }
          }
        }
    if (MODE == 0) {
      cnt[id] = c;
    } else {
      // sort this droplet's run by partner id (insertion sort; runs are short)
      const long long b0 = off[id];
      const long long b1 = o_end < cap ? o_end : cap;
      for (long long x = b0 + 1; x < b1; ++x) {
        const int v = pairs[2 * x + 1];
        long long y = x - 1;
        while (y >= b0 && pairs[2 * y + 1] > v) { pairs[2 * (y + 1) + 1] = pairs[2 * y + 1]; --y; }
        pairs[2 * (y + 1) + 1] = v;
      }
    }
  }
}

__global__ void k_finish(const unsigned* __restrict__ off, long long n, long long cap, int64_t* __restrict__ count,
                         unsigned* __restrict__ status) {
  const long long tot = off[n];
  *count = tot;
  if (tot > cap && status) atomicOr(status, LD_STATUS_PAIR_OVERFLOW);
}

inline int gridn(long long n, int th) {
  long long b = (n + th - 1) / th;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

struct ld_collider {
  long long nmax = 0;
  int nc = 0;
  unsigned *key = nullptr, *val = nullptr, *key2 = nullptr, *val2 = nullptr, *hist = nullptr, *cnt = nullptr;
  int *start = nullptr, *end = nullptr;
  double4* sp = nullptr;
  unsigned* status = nullptr;
  int nblocks = 0;
};

extern "C" {

int ld_collider_create(ld_collider** out, int64_t nmax, int32_t nc) {
  if (!out || nmax < 1 || nmax > (1LL << 31) - 2 || nc < 1 || (long long)nc * nc * nc > (1LL << 31))
    return ld_fail(LD_ERR_ARG, "ld_collider_create: bad arguments");
  *out = nullptr;
  ld_collider* c = new (std::nothrow) ld_collider();
  if (!c) return ld_fail(LD_ERR_NOMEM, "host allocation failed");
  c->nmax = nmax;
  c->nc = nc;
  c->nblocks = (int)((nmax + RS_TILE - 1) / RS_TILE);
  const long long ncell = (long long)nc * nc * nc;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
  A((void**)&c->key, 4 * nmax);
  A((void**)&c->val, 4 * nmax);
  A((void**)&c->key2, 4 * nmax);
  A((void**)&c->val2, 4 * nmax);
  A((void**)&c->hist, 4 * (size_t)RADIX * c->nblocks);
  A((void**)&c->cnt, 4 * (nmax + 1));
  A((void**)&c->start, 4 * ncell);
  A((void**)&c->end, 4 * ncell);
  A((void**)&c->sp, sizeof(double4) * nmax);
  A((void**)&c->status, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(c->status, 0, sizeof(unsigned));
  if (e != cudaSuccess) {
    ld_set_last_error(e);
    ld_collider_destroy(c);
    return LD_ERR_CUDA;
  }
  *out = c;
  return LD_OK;
}

int ld_collider_destroy(ld_collider* c) {
  if (!c) return LD_OK;
  cudaFree(c->key); cudaFree(c->val); cudaFree(c->key2); cudaFree(c->val2); cudaFree(c->hist);
  cudaFree(c->cnt); cudaFree(c->start); cudaFree(c->end); cudaFree(c->sp); cudaFree(c->status);
  delete c;
  return LD_OK;
}

int ld_radix_sort_u32(ld_collider* c, unsigned* key, unsigned* val, int64_t n, int bits, void* stream) {
  if (!c || !key || !val || n < 0 || n > c->nmax || bits < 1 || bits > 32)
    return ld_fail(LD_ERR_ARG, "ld_radix_sort_u32: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return LD_OK;
  const int nb = (int)((n + RS_TILE - 1) / RS_TILE);
  unsigned *ki = key, *vi = val, *ko = c->key2, *vo = c->val2;
  const int passes = (bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    k_rs_hist<<<nb, RS_THREADS, 0, s>>>(ki, n, 8 * p, c->hist, nb);
    k_scan_u32<<<1, 1024, 0, s>>>(c->hist, (long long)RADIX * nb);
    k_rs_scatter<<<nb, RS_THREADS, 0, s>>>(ki, vi, ko, vo, n, 8 * p, c->hist, nb);
    unsigned* t;
    t = ki; ki = ko; ko = t;
    t = vi; vi = vo; vo = t;
  }
  if (ki != key) {  // odd number of passes: result is in the scratch pair
    LD_CUDA_CHECK(cudaMemcpyAsync(key, ki, 4 * n, cudaMemcpyDeviceToDevice, s));
    LD_CUDA_CHECK(cudaMemcpyAsync(val, vi, 4 * n, cudaMemcpyDeviceToDevice, s));
  }
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_collide(ld_collider* c, const double* pos, const double* radius, int64_t n, double L, int32_t* pairs,
               int64_t cap, int64_t* count, void* stream) {
  if (!c || !pos || !radius || !count || n < 0 || n > c->nmax || cap < 0 || (cap > 0 && !pairs) || !(L > 0))
    return ld_fail(LD_ERR_ARG, "ld_collide: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = c->nc;
  const double cw = L / nc;
  const long long ncell = (long long)nc * nc * nc;
  if (n == 0) {
    LD_CUDA_CHECK(cudaMemsetAsync(count, 0, sizeof(int64_t), s));
    return LD_OK;
  }
  k_cell_keys<<<gridn(n, 256), 256, 0, s>>>(pos, n, L, cw, nc, c->key, c->val);
  int bits = 1;
  while ((1LL << bits) < ncell) ++bits;
  if (int rc = ld_radix_sort_u32(c, c->key, c->val, n, bits, stream)) return rc;
  LD_CUDA_CHECK(cudaMemsetAsync(c->start, 0, 4 * ncell, s));
  LD_CUDA_CHECK(cudaMemsetAsync(c->end, 0, 4 * ncell, s));
  k_cell_ranges<<<gridn(n, 256), 256, 0, s>>>(c->key, n, c->start, c->end);
  k_sorted_copy<<<gridn(n, 256), 256, 0, s>>>(pos, radius, c->val, n, L, c->sp);
  k_pairs<0><<<gridn(n, 128), 128, 0, s>>>(c->sp, c->val, c->key, c->start, c->end, n, nc, L, c->cnt, nullptr,
                                           nullptr, 0);
  LD_CUDA_CHECK(cudaMemsetAsync(c->cnt + n, 0, 4, s));
  k_scan_u32<<<1, 1024, 0, s>>>(c->cnt, n + 1);
  k_pairs<1><<<gridn(n, 128), 128, 0, s>>>(c->sp, c->val, c->key, c->start, c->end, n, nc, L, nullptr, c->cnt,
                                           pairs, cap);
  k_finish<<<1, 1, 0, s>>>(c->cnt, n, cap, count, c->status);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_collider_status(ld_collider* c, uint32_t* flags, int clear, void* stream) {
  if (!c || !flags) return ld_fail(LD_ERR_ARG, "ld_collider_status: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned h = 0;
  LD_CUDA_CHECK(cudaMemcpyAsync(&h, c->status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  LD_CUDA_CHECK(cudaStreamSynchronize(s));
  if (clear) LD_CUDA_CHECK(cudaMemsetAsync(c->status, 0, sizeof(unsigned), s));
  *flags = h;
  return LD_OK;
}

int ld_collider_sorted(ld_collider* c, const uint32_t** keys, const uint32_t** ids) {
  if (!c) return ld_fail(LD_ERR_ARG, "ld_collider_sorted: null collider");
  if (keys) *keys = c->key;
  if (ids) *ids = c->val;
  return LD_OK;
}

}  // extern "C"
