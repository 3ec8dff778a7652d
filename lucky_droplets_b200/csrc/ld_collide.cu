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

// Multi-block exclusive scan, phase 1: each block scans a tile of SCAN_TILE counts in place and
// writes the tile total to sums[blockIdx.x].
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER;

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_tiles(unsigned* __restrict__ a, long long m, unsigned* __restrict__ sums) {
  __shared__ unsigned buf[SCAN_TILE];
  __shared__ unsigned wsum[SCAN_THREADS / 32];
  const long long base = (long long)blockIdx.x * SCAN_TILE;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  for (int i = t; i < SCAN_TILE; i += SCAN_THREADS) buf[i] = base + i < m ? a[base + i] : 0u;
  __syncthreads();
  unsigned v[SCAN_PER];
  unsigned run = 0;
#pragma unroll
  for (int q = 0; q < SCAN_PER; ++q) { v[q] = run; run += buf[t * SCAN_PER + q]; }
  // inclusive scan of the per-thread totals: warp shuffles, then warp totals
  unsigned x = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned ws = lane < SCAN_THREADS / 32 ? wsum[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    if (lane < SCAN_THREADS / 32) wsum[lane] = ws;
  }
  __syncthreads();
  const unsigned before = (x - run) + (w ? wsum[w - 1] : 0u);
#pragma unroll
  for (int q = 0; q < SCAN_PER; ++q) buf[t * SCAN_PER + q] = before + v[q];
  if (t == SCAN_THREADS - 1) sums[blockIdx.x] = before + run;
  __syncthreads();
  for (int i = t; i < SCAN_TILE; i += SCAN_THREADS)
    if (base + i < m) a[base + i] = buf[i];
}

// phase 3: add the scanned tile totals
__global__ void k_scan_add(unsigned* __restrict__ a, long long m, const unsigned* __restrict__ sums) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) a[i] += sums[i / SCAN_TILE];
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

// MODE 0: count partners per droplet id; MODE 1: emit pairs.  DEDUP: nc < 3, where the 27
// neighbour offsets can name the same cell more than once.
template <int MODE, bool DEDUP>
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
          if (DEDUP) {
            bool dup = false;
            for (int q = 0; q < ns; ++q) dup |= seen[q] == nk;
            if (dup) continue;
            seen[ns++] = nk;
          }
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

// Warp per cell (nc >= 3): the cell against itself and its 13 forward neighbours (offsets after
// (0,0,0) in lexicographic order), so every unordered droplet pair is tested exactly once.  Pairs
// are visited in a fixed order (neighbour, then i-major pair index in chunks of 32) and hits are
// ranked inside each chunk by ballot, so the emitted order is deterministic.
// MODE 0: cnt[cell] = hits; MODE 1: emit at off[cell] + rank as (min index, max index).
template <int MODE>
__global__ void __launch_bounds__(256)
k_cell_pairs(const double4* __restrict__ sp, const int* __restrict__ start, const int* __restrict__ end, int nc,
             double L, unsigned* __restrict__ cnt, const unsigned* __restrict__ off, int* __restrict__ pairs,
             long long cap) {
  const int lane = threadIdx.x & 31;
  const long long ncell = (long long)nc * nc * nc;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); c < ncell; c += warps) {
    const int cz = (int)(c % nc), cy = (int)((c / nc) % nc), cx = (int)(c / ((long long)nc * nc));
    const int a0 = start[c], a1 = end[c];
    const int na = a1 - a0;
    unsigned hits = 0;
    long long o = MODE == 1 ? (long long)off[c] : 0;
    if (na > 0) {
      for (int q = 0; q < 14; ++q) {
        // q = 0: the cell itself; q = 1..13: forward offsets
        int dx = 0, dy = 0, dz = 0;
        if (q > 0) {
          const int r = q + 13;  // offsets -1..1 enumerated as r = (dx+1)*9 + (dy+1)*3 + (dz+1), r > 13
          dx = r / 9 - 1;
          dy = (r / 3) % 3 - 1;
          dz = r % 3 - 1;
        }
        const long long nb = ((long long)((cx + dx + nc) % nc) * nc + (cy + dy + nc) % nc) * nc + (cz + dz + nc) % nc;
        const int b0 = start[nb], b1 = end[nb];
        const int nbb = b1 - b0;
        const long long npair = (long long)na * nbb;
        for (long long base = 0; base < npair; base += 32) {
          const long long pidx = base + lane;
          bool hit = false;
          int ia = 0, ib = 0;
          if (pidx < npair) {
            ia = a0 + (int)(pidx / nbb);
            ib = b0 + (int)(pidx % nbb);
            if (q > 0 || ib > ia) hit = overlap(sp[ia], sp[ib], L);
          }
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (MODE == 1 && hit) {
            const long long dst = o + __popc(m & ((1u << lane) - 1u));
            if (dst < cap) {
              pairs[2 * dst] = ia < ib ? ia : ib;
              pairs[2 * dst + 1] = ia < ib ? ib : ia;
            }
          }
          o += __popc(m);
          hits += __popc(m);
        }
      }
    }
    if (MODE == 0 && lane == 0) cnt[c] = hits;
  }
}

// sorted-array indices -> droplet indices, (i, j) with i < j
__global__ void k_map_pairs(const unsigned* __restrict__ total, long long cap, const unsigned* __restrict__ sval,
                            int* __restrict__ pairs) {
  const long long m = (long long)*total < cap ? (long long)*total : cap;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x) {
    const int a = (int)sval[pairs[2 * e]], b = (int)sval[pairs[2 * e + 1]];
    pairs[2 * e] = a < b ? a : b;
    pairs[2 * e + 1] = a < b ? b : a;
  }
}

__global__ void k_finish(const unsigned* __restrict__ off, long long n, long long cap, int64_t* __restrict__ count,
                         unsigned* __restrict__ status) {
  const long long tot = off[n];
  *count = tot;
  if (tot > cap && status) atomicOr(status, LD_STATUS_PAIR_OVERFLOW);
}

// dst row i = src row order[i]; rows of `words` 32-bit words.
__global__ void k_permute_rows(const unsigned* __restrict__ src, unsigned* __restrict__ dst,
                               const unsigned* __restrict__ order, long long n, int words) {
  const long long total = n * (long long)words;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / words;
    const int w = (int)(e - i * words);
    dst[e] = src[(long long)order[i] * words + w];
  }
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
  unsigned* sums = nullptr;  // scan tile totals
  int nblocks = 0;
  ld_plan* trace = nullptr;  // plan whose event trace records this collider's launches
};

namespace {
// Exclusive scan of m counts in place (m <= SCAN_TILE^2).
int scan_u32(ld_collider* c, unsigned* a, long long m, cudaStream_t s) {
  const long long tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
  if (tiles > SCAN_TILE) return ld_fail(LD_ERR_UNSUPPORTED, "scan of %lld elements", m);
  k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(a, m, c->sums);
  if (tiles > 1) {
    unsigned* sums2 = c->sums + tiles;
    k_scan_tiles<<<1, SCAN_THREADS, 0, s>>>(c->sums, tiles, sums2);
    k_scan_add<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(a, m, c->sums);
  }
  LD_LAUNCH_CHECK();
  return LD_OK;
}
}  // namespace

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
  A((void**)&c->cnt, 4 * ((nmax > ncell ? nmax : ncell) + 1));
  A((void**)&c->start, 4 * ncell);
  A((void**)&c->end, 4 * ncell);
  A((void**)&c->sp, sizeof(double4) * nmax);
  A((void**)&c->status, sizeof(unsigned));
  {
    long long m = (nmax + 1) > (long long)RADIX * c->nblocks ? (nmax + 1) : (long long)RADIX * c->nblocks;
    if (ncell + 1 > m) m = ncell + 1;
    A((void**)&c->sums, 4 * ((m + SCAN_TILE - 1) / SCAN_TILE + 2));
  }
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
  cudaFree(c->sums);
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
    if (int rc = scan_u32(c, c->hist, (long long)RADIX * nb, s)) return rc;
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
  if (!c || !count || n < 0 || n > c->nmax || cap < 0 || !(L > 0) || (n > 0 && (!pos || !radius)) ||
      (n > 0 && cap > 0 && !pairs))
    return ld_fail(LD_ERR_ARG, "ld_collide: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = c->nc;
  const double cw = L / nc;
  const long long ncell = (long long)nc * nc * nc;
  if (n == 0) {
    LD_CUDA_CHECK(cudaMemsetAsync(count, 0, sizeof(int64_t), s));
    return LD_OK;
  }
  {
    ProfScope ps(c->trace, KID_COLL_SORT, s);
    k_cell_keys<<<gridn(n, 256), 256, 0, s>>>(pos, n, L, cw, nc, c->key, c->val);
    int bits = 1;
    while ((1LL << bits) < ncell) ++bits;
    if (int rc = ld_radix_sort_u32(c, c->key, c->val, n, bits, stream)) return rc;
  }
  ProfScope ps(c->trace, KID_COLL_PAIRS, s);
  LD_CUDA_CHECK(cudaMemsetAsync(c->start, 0, 4 * ncell, s));
  LD_CUDA_CHECK(cudaMemsetAsync(c->end, 0, 4 * ncell, s));
  k_cell_ranges<<<gridn(n, 256), 256, 0, s>>>(c->key, n, c->start, c->end);
  k_sorted_copy<<<gridn(n, 256), 256, 0, s>>>(pos, radius, c->val, n, L, c->sp);
  if (nc >= 3) {
    // cell-pair search over sorted positions; pairs come out as sorted-array indices and are
    // mapped back to droplet indices by k_map_pairs
    const int gw = gridn(ncell * 32, 256);
    k_cell_pairs<0><<<gw, 256, 0, s>>>(c->sp, c->start, c->end, nc, L, c->cnt, nullptr, nullptr, 0);
    LD_CUDA_CHECK(cudaMemsetAsync(c->cnt + ncell, 0, 4, s));
    if (int rc = scan_u32(c, c->cnt, ncell + 1, s)) return rc;
    k_cell_pairs<1><<<gw, 256, 0, s>>>(c->sp, c->start, c->end, nc, L, nullptr, c->cnt, pairs, cap);
    k_map_pairs<<<gridn(cap, 256), 256, 0, s>>>(c->cnt + ncell, cap, c->val, pairs);
    k_finish<<<1, 1, 0, s>>>(c->cnt, ncell, cap, count, c->status);
  } else {
    k_pairs<0, true><<<gridn(n, 128), 128, 0, s>>>(c->sp, c->val, c->key, c->start, c->end, n, nc, L, c->cnt,
                                                   nullptr, nullptr, 0);
    LD_CUDA_CHECK(cudaMemsetAsync(c->cnt + n, 0, 4, s));
    if (int rc = scan_u32(c, c->cnt, n + 1, s)) return rc;
    k_pairs<1, true><<<gridn(n, 128), 128, 0, s>>>(c->sp, c->val, c->key, c->start, c->end, n, nc, L, nullptr,
                                                   c->cnt, pairs, cap);
    k_finish<<<1, 1, 0, s>>>(c->cnt, n, cap, count, c->status);
  }
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_cell_order(ld_collider* c, const double* pos, int64_t n, double L, uint32_t* order, void* stream) {
  if (!c || n < 0 || n > c->nmax || !(L > 0) || (n > 0 && (!pos || !order)))
    return ld_fail(LD_ERR_ARG, "ld_cell_order: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  ProfScope ps(c->trace, KID_CELL_ORDER, s);
  const int nc = c->nc;
  const long long ncell = (long long)nc * nc * nc;
  k_cell_keys<<<gridn(n, 256), 256, 0, s>>>(pos, n, L, L / nc, nc, c->key, c->val);
  int bits = 1;
  while ((1LL << bits) < ncell) ++bits;
  if (int rc = ld_radix_sort_u32(c, c->key, c->val, n, bits, stream)) return rc;
  LD_CUDA_CHECK(cudaMemcpyAsync(order, c->val, 4 * n, cudaMemcpyDeviceToDevice, s));
  return LD_OK;
}

int ld_permute_rows(const void* src, void* dst, const uint32_t* order, int64_t n, int32_t row_bytes, void* stream) {
  if (n < 0 || row_bytes <= 0 || (row_bytes % 4) != 0 || (n > 0 && (!src || !dst || !order)) || src == dst)
    return ld_fail(LD_ERR_ARG, "ld_permute_rows: bad arguments (row_bytes must be a positive multiple of 4, src != dst)");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int words = row_bytes / 4;
  const long long total = n * (long long)words;
  k_permute_rows<<<gridn(total, 256), 256, 0, s>>>((const unsigned*)src, (unsigned*)dst, order, n, words);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_collider_trace(ld_collider* c, ld_plan* plan) {
  if (!c) return ld_fail(LD_ERR_ARG, "ld_collider_trace: null collider");
  c->trace = plan;
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
