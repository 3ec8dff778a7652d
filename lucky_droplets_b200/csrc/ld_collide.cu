// Cell-list collision detection, the counting sort by cell it uses, and a stable LSD radix sort.
//
// Pipeline (one call of ld_collide):
//   sort      counting sort by cell: key[i] = cell of the wrapped position of droplet i;
//             occupancies by atomics, cs[k] = first sorted index of cell k (k = 0..ncell,
//             cs[ncell] = n) by a scan, an unordered scatter, then every droplet placed at its
//             cell's start plus its rank by index within the cell, which is exactly the order of a
//             stable sort of (key, i); sorted copies of the wrapped positions and radii (FP64,
//             and an FP32 copy for the pre-test) written alongside.  (More than 2^24 cells: LSD
//             radix sort with 8-bit digits and binary-searched starts instead.)
//   count     per sorted droplet: partners among the cell itself and its 13 forward neighbours
//             (the first KEEP of them recorded)
//   scan      exclusive scan of the counts in sorted order -> offsets, total
//   wide      droplets with 2 r > cell width ("wide"; none when the cell width is at least twice
//             the largest radius) also search the cells within 2 r of them for the partners
//             with ri + rj > cell width, which the neighbour search leaves out: counted by the
//             block of the column visit that meets them, emitted by the block of the emit pass
//   emit      pairs at offset + t in the fixed visiting order (copied from the record, or searched
//             again for droplets with more partners), then mapped to droplet ids (i < j)
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

// Cell keys of a multi-box collider: box b's cells come after those of boxes 0..b-1 (box = null:
// one box).
__device__ __forceinline__ unsigned box_base(const int* __restrict__ box, long long i, int nc) {
  return box ? (unsigned)box[i] * (unsigned)nc * (unsigned)nc * (unsigned)nc : 0u;
}

__global__ void k_cell_keys(const double* __restrict__ pos, long long n, double L, double cw, int nc,
                            unsigned* __restrict__ key, unsigned* __restrict__ val, const int* __restrict__ box) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cx = cell_of(wrapL(pos[3 * i], L), cw, nc);
    const int cy = cell_of(wrapL(pos[3 * i + 1], L), cw, nc);
    const int cz = cell_of(wrapL(pos[3 * i + 2], L), cw, nc);
    key[i] = box_base(box, i, nc) + (unsigned)((cx * nc + cy) * nc + cz);
    val[i] = (unsigned)i;
  }
}

// ---- counting sort by cell (the sort of ld_collide) -------------------------------------------
__global__ void k_cell_count(const double* __restrict__ pos, long long n, double L, double cw, int nc,
                             unsigned* __restrict__ key, unsigned* __restrict__ rank, unsigned* __restrict__ occ,
                             const int* __restrict__ box) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cx = cell_of(wrapL(pos[3 * i], L), cw, nc);
    const int cy = cell_of(wrapL(pos[3 * i + 1], L), cw, nc);
    const int cz = cell_of(wrapL(pos[3 * i + 2], L), cw, nc);
    const unsigned k = box_base(box, i, nc) + (unsigned)((cx * nc + cy) * nc + cz);
    key[i] = k;
    rank[i] = atomicAdd(&occ[k], 1u);  // arrival order: unordered
  }
}

__global__ void k_cell_scatter(const unsigned* __restrict__ key, const unsigned* __restrict__ rank,
                               const int* __restrict__ cs, long long n, unsigned* __restrict__ run) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    run[cs[key[i]] + rank[i]] = (unsigned)i;
}

// Sorted copies of one sorted slot: cell key, wrapped FP64 position + radius, FP32 copy.
__device__ __forceinline__ void sorted_slot(long long s, unsigned k, unsigned i, const double* __restrict__ pos,
                                            const double* __restrict__ rad, double L, unsigned* __restrict__ skey,
                                            double4* __restrict__ sp, float4* __restrict__ spf) {
  double4 q;
  q.x = wrapL(pos[3 * (long long)i], L);
  q.y = wrapL(pos[3 * (long long)i + 1], L);
  q.z = wrapL(pos[3 * (long long)i + 2], L);
  q.w = rad[i];
  skey[s] = k;
  sp[s] = q;
  spf[s] = make_float4((float)q.x, (float)q.y, (float)q.z, (float)q.w);
}

constexpr int kSmallCell = 64;  // cells up to this occupancy are placed by rank counting

// Thread per droplet (index order): its place in the sorted order is its cell's start plus the
// number of the cell's droplets with a smaller index, counted over the cell's unordered run;
// writes the sorted index, key and copies there.  Cells above kSmallCell droplets are left to
// k_cell_big (the droplet in the run's first slot appends the cell to `big`).
__global__ void k_cell_place(const unsigned* __restrict__ key, const int* __restrict__ cs,
                             const unsigned* __restrict__ run, long long n, const double* __restrict__ pos,
                             const double* __restrict__ rad, double L, unsigned* __restrict__ sval,
                             unsigned* __restrict__ skey, double4* __restrict__ sp, float4* __restrict__ spf,
                             unsigned* __restrict__ big, unsigned* __restrict__ nbig) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned k = key[i];
    const int s0 = cs[k], s1 = cs[k + 1];
    if (s1 - s0 > kSmallCell) {
      if (run[s0] == (unsigned)i) big[atomicAdd(nbig, 1u)] = k;
      continue;
    }
    int r = 0;
    for (int j = s0; j < s1; ++j) r += run[j] < (unsigned)i ? 1 : 0;
    const int s = s0 + r;
    sval[s] = (unsigned)i;
    sorted_slot(s, k, (unsigned)i, pos, rad, L, skey, sp, spf);
  }
}

// Block per large cell (grid-stride over the list): a bitonic network in global memory over the
// cell's unordered run (virtual +inf padding to a power of two; every compare-exchange puts the
// smaller index first, so padded slots never move), then the sorted index, key and copies.
__global__ void __launch_bounds__(512)
k_cell_big(const int* __restrict__ cs, const unsigned* __restrict__ big, const unsigned* __restrict__ nbig,
           unsigned* __restrict__ run, const double* __restrict__ pos, const double* __restrict__ rad, double L,
           unsigned* __restrict__ sval, unsigned* __restrict__ skey, double4* __restrict__ sp, float4* __restrict__ spf) {
  const unsigned nb = *nbig;
  for (unsigned b = blockIdx.x; b < nb; b += gridDim.x) {
    const unsigned k = big[b];
    const int s0 = cs[k], m = cs[k + 1] - s0;
    unsigned* v = run + s0;
    int P = 1;
    while (P < m) P <<= 1;
    for (int kk = 2; kk <= P; kk <<= 1) {
      for (int d = kk >> 1; d >= 1; d >>= 1) {
        for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
          const int i = ((t & ~(d - 1)) << 1) | (t & (d - 1));  // insert a 0 bit at position log2(d)
          const int j = d == (kk >> 1) ? (i ^ (kk - 1)) : (i | d);  // flip step first, then half-cleaners
          if (j < m) {
            const unsigned x = v[i], y = v[j];
            if (x > y) { v[i] = y; v[j] = x; }
          }
        }
        __syncthreads();
      }
    }
    for (int x = threadIdx.x; x < m; x += blockDim.x) {
      sval[s0 + x] = v[x];
      sorted_slot(s0 + x, k, v[x], pos, rad, L, skey, sp, spf);
    }
    __syncthreads();
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

// ---- cell starts and sorted copies ------------------------------------------------------------
// cs[k] = number of sorted keys < k, for k = 0..ncell (binary search; cells are balanced work).
__global__ void k_cell_starts(const unsigned* __restrict__ skey, long long n, long long ncell, int* __restrict__ cs) {
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

__global__ void k_sorted_copy(const double* __restrict__ pos, const double* __restrict__ rad,
                              const unsigned* __restrict__ sval, long long n, double L, double4* __restrict__ sp,
                              float4* __restrict__ spf) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const unsigned i = sval[s];
    double4 q;
    q.x = wrapL(pos[3 * (long long)i], L);
    q.y = wrapL(pos[3 * (long long)i + 1], L);
    q.z = wrapL(pos[3 * (long long)i + 2], L);
    q.w = rad[i];
    sp[s] = q;
    spf[s] = make_float4((float)q.x, (float)q.y, (float)q.z, (float)q.w);
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

// The pairs the neighbour-cell search reports: overlapping with ri + rj <= cw (always true when
// cw >= 2 max radius; the others are found by the wide droplets' search).
__device__ __forceinline__ bool overlap_near(const double4 a, const double4 b, double L, double cw) {
  return !(__dadd_rn(a.w, b.w) > cw) && overlap(a, b, L);
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
    const int nc3 = nc * nc * nc;
    const int key = (int)skey[s];
    const int kb = (key / nc3) * nc3;  // the box's first cell
    const int cz = key % nc, cy = (key / nc) % nc, cx = (key / (nc * nc)) % nc;
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
          const int nk = kb + (nx * nc + ny) * nc + nz;
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

// FP32 pre-test of the FP64 rule: true whenever overlap() is.  Coordinates in [0, L) rounded
// to FP32 are off by at most L 2^-24 each, so every float difference is within 1.2e-7 L of the
// FP64 one and the distance within 2.1e-7 L (plus relative roundoff of 1e-7 of the distance);
// the margin of 1e-6 (L + rs) covers both several times over.
__device__ __forceinline__ bool near_f(const float4 a, const float4 b, float L, float h, float margin) {
  float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  if (dx > h) dx -= L;
  if (dx < -h) dx += L;
  if (dy > h) dy -= L;
  if (dy < -h) dy += L;
  if (dz > h) dz -= L;
  if (dz < -h) dz += L;
  const float r = a.w + b.w + margin;
  return dx * dx + dy * dy + dz * dz < r * r;
}

// Block per (cell column (cx, cy), part), nc >= 3; thread per droplet of the column (the part's
// share of them).  Its partners are searched among the cell itself (partners after it in the
// sorted order) and the 13 forward neighbours, visited in a fixed order r = 0..13:
//   r = 0: the cell itself; r = 1: (0, 0, +1); r = 2..13: columns q = 1..4 (offsets (0,+1),
//   (+1,-1), (+1,0), (+1,+1)) at dz = -1, 0, +1,
// and in sorted order inside each target cell, so every unordered pair is tested exactly once.
// The five columns' cell starts, their periodic shifts and (when they fit in cap_smem rows) their
// FP32 positions are staged in shared memory; the home cell comes from the sorted key and the
// neighbour cells by compare-and-wrap, so the visit needs no integer division.  The periodic
// image of a neighbour cell is fixed (a colliding pair is closer than one cell, nc >= 3): the
// home position is shifted once per target cell; a wrong image only lengthens the distance (the
// FP64 rule decides).  Each droplet stores its partner count and its first KEEP partners (sorted
// indices) in scr; k_emit_pairs writes the pairs from the scanned counts, searching again only
// for droplets with more than KEEP partners.
constexpr int COL_THREADS = 256;
constexpr int KEEP = 16;  // partners recorded per droplet (more: searched again by k_emit_pairs)
constexpr int kColSmemRows = 12288;  // 192 KB of staged FP32 rows per block at most

__device__ __forceinline__ void col_offset(int q, int& ox, int& oy) {
  ox = q < 2 ? 0 : 1;
  oy = q == 0 ? 0 : (q == 1 ? 1 : q - 3);
}

// The visit of one droplet (sorted index i, t-th of its column); STAGED: positions from colbuf.
// Returns whether the droplet is wide (2 r > cw: its partners beyond the neighbour cells are
// counted by the block afterwards).
template <bool STAGED>
__device__ __forceinline__ bool col_visit(int i, int t, const double4* __restrict__ sp, const float4* __restrict__ spf,
                                          const float4* colbuf, const int* cst, const int* dl, const float* shx,
                                          const float* shy, int cz, int nc, double L, double cw, float Lf,
                                          float margin, unsigned* __restrict__ cnt, int* __restrict__ scr) {
  const float4 mf = STAGED ? colbuf[t] : spf[i];
  const float mar = margin + 1e-6f * mf.w;
  unsigned c = 0;
  // away from the z faces the three cells z-1, z, z+1 of a column are one contiguous sorted range
  // with no periodic shift along z: 5 ranges (the own column from i + 1 through cell z + 1, then
  // the four forward columns), visited in exactly the order of the 14 cells
  const bool interior = cz >= 1 && cz <= nc - 2;
  const int nseg = interior ? 5 : 14;
#pragma unroll 1
  for (int r = 0; r < nseg; ++r) {
    int q, g0, g1;
    float sz;
    if (interior) {
      q = r;
      sz = 0.f;
      g0 = r == 0 ? i + 1 : cst[q * (nc + 1) + cz - 1];
      g1 = cst[q * (nc + 1) + cz + 2];
    } else {
      q = r < 2 ? 0 : 1 + (r - 2) / 3;
      const int dz = r < 2 ? r : (r - 2) % 3 - 1;
      const int zr = cz + dz;
      const int zz = zr < 0 ? zr + nc : (zr >= nc ? zr - nc : zr);
      sz = zr >= nc ? -Lf : (zr < 0 ? Lf : 0.f);
      g0 = r == 0 ? i + 1 : cst[q * (nc + 1) + zz];
      g1 = cst[q * (nc + 1) + zz + 1];
    }
    const float ax = mf.x + shx[q], ay = mf.y + shy[q], az = mf.z + sz;
    const int d = dl[q];
    // two candidates at a time on packed FP32 pairs (each half rounds as the scalar operation);
    // b - a instead of a - b: the squares are the same
    const float2 nax = make_float2(-ax, -ax), nay = make_float2(-ay, -ay), naz = make_float2(-az, -az);
    const float2 mw = make_float2(mf.w, mf.w), mr = make_float2(mar, mar);
    int g = g0;
    for (; g + 1 < g1; g += 2) {
      const float4 b0 = STAGED ? colbuf[g - d] : spf[g];
      const float4 b1 = STAGED ? colbuf[g + 1 - d] : spf[g + 1];
      const float2 dx = __fadd2_rn(make_float2(b0.x, b1.x), nax), dy = __fadd2_rn(make_float2(b0.y, b1.y), nay),
                   dz = __fadd2_rn(make_float2(b0.z, b1.z), naz);
      const float2 rr = __fadd2_rn(__fadd2_rn(mw, make_float2(b0.w, b1.w)), mr);
      const float2 d2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
      const float2 r2 = __fmul2_rn(rr, rr);
      if (d2.x < r2.x && overlap_near(sp[i], sp[g], L, cw)) {
        if (c < KEEP) scr[(long long)KEEP * i + c] = g;
        ++c;
      }
      if (d2.y < r2.y && overlap_near(sp[i], sp[g + 1], L, cw)) {
        if (c < KEEP) scr[(long long)KEEP * i + c] = g + 1;
        ++c;
      }
    }
    if (g < g1) {
      const float4 b = STAGED ? colbuf[g - d] : spf[g];
      const float dxf = ax - b.x, dyf = ay - b.y, dzf = az - b.z;
      const float rr = mf.w + b.w + mar;
      if (dxf * dxf + dyf * dyf + dzf * dzf < rr * rr && overlap_near(sp[i], sp[g], L, cw)) {
        if (c < KEEP) scr[(long long)KEEP * i + c] = g;
        ++c;
      }
    }
  }
  cnt[i] = c;
  // FP32 radius first (rounding is monotone: r > cw / 2 implies float(r) >= float(cw / 2))
  return mf.w >= (float)(0.5 * cw) && sp[i].w > 0.5 * cw;
}

// ---- wide droplets ------------------------------------------------------------------------------
// A pair with ri + rj > cw (cw the cell width) has at least one droplet with 2 r > cw, a wide
// droplet.  It is reported once, by its owner: the droplet of larger radius (equal radii: the
// smaller sorted index), which is wide.  The owner s searches every cell within R = floor(2 rs /
// cw) + 1 cells of its own along each axis (all nc when 2 R + 1 >= nc), since its partner is closer
// than rs + rt <= 2 rs.  The owner's pairs follow the pairs of its neighbour-cell search in its
// run of the output.  Work items of a wide droplet: the 14 cells of the neighbour search (emit
// only), then the cells of the wide search in (x, y, z) order; the block that meets a wide droplet
// (the column visit for the count, the emit pass for the pairs) takes its items in contiguous
// runs, one run per thread, counts, scans the counts and writes, so the order is that of a serial
// visit.

struct WideCell {
  long long kb;  // the box's first cell
  int cx, cy, cz, R, ax;  // home cell, reach, cells per axis visited
};

__device__ __forceinline__ WideCell wide_cell(unsigned key, int nc, double r, double cw) {
  WideCell w;
  const unsigned nc3 = (unsigned)nc * nc * nc;
  w.kb = (long long)(key / nc3) * nc3;
  w.cz = (int)(key % (unsigned)nc);
  w.cy = (int)((key / nc) % nc);
  w.cx = (int)((key / ((unsigned)nc * nc)) % nc);
  const double rr = floor(__ddiv_rn(__dadd_rn(r, r), cw));
  w.R = rr < (double)nc ? (int)rr + 1 : nc;
  w.ax = 2 * w.R + 1 >= nc ? nc : 2 * w.R + 1;
  return w;
}

// Visit work item `it` of wide droplet s: WRITE 0 counts, 1 writes at pairs[o...]; returns the hits.
template <bool WRITE>
__device__ unsigned wide_item(int it, bool with_near, int s, const WideCell& w, const double4& me, const float4& mf,
                              const double4* __restrict__ sp, const float4* __restrict__ spf, const int* __restrict__ cs,
                              int nc, double L, double cw, float Lf, float hf, float mar, int* __restrict__ pairs,
                              long long o, long long cap) {
  unsigned c = 0;
  if (with_near && it < 14) {  // the neighbour search of k_emit_pairs, segment r = it
    const int r = it;
    const int q = r < 2 ? 0 : 1 + (r - 2) / 3;
    const int dz = r < 2 ? r : (r - 2) % 3 - 1;
    const int z = (w.cz + dz + nc) % nc;
    const int ox = q < 2 ? 0 : 1;
    const int oy = q == 0 ? 0 : (q == 1 ? 1 : q - 3);
    const long long k = w.kb + ((long long)((w.cx + ox) % nc) * nc + (w.cy + oy + nc) % nc) * nc + z;
    const int g1 = cs[k + 1];
    for (int g = r == 0 ? s + 1 : cs[k]; g < g1; ++g) {
      if (!near_f(mf, spf[g], Lf, hf, mar)) continue;
      if (!overlap_near(me, sp[g], L, cw)) continue;
      if (WRITE && o + c < cap) { pairs[2 * (o + c)] = s; pairs[2 * (o + c) + 1] = g; }
      ++c;
    }
    return c;
  }
  const int m = with_near ? it - 14 : it;
  const int wz = m % w.ax, wy = (m / w.ax) % w.ax, wx = m / (w.ax * w.ax);
  const int x = w.ax == nc ? wx : (w.cx - w.R + wx + nc) % nc;
  const int y = w.ax == nc ? wy : (w.cy - w.R + wy + nc) % nc;
  const int z = w.ax == nc ? wz : (w.cz - w.R + wz + nc) % nc;
  const long long k = w.kb + ((long long)x * nc + y) * nc + z;
  const int g1 = cs[k + 1];
  for (int g = cs[k]; g < g1; ++g) {
    if (g == s || !near_f(mf, spf[g], Lf, hf, mar)) continue;
    const double4 b = sp[g];
    if (!(__dadd_rn(me.w, b.w) > cw)) continue;  // reported by the neighbour search
    if (b.w > 0.5 * cw && (b.w > me.w || (b.w == me.w && g < s))) continue;  // g owns the pair
    if (!overlap(me, b, L)) continue;
    if (WRITE && o + c < cap) { pairs[2 * (o + c)] = s; pairs[2 * (o + c) + 1] = g; }
    ++c;
  }
  return c;
}

// Block-wide exclusive scan of one count per thread (NTH threads, all of them calling); returns
// the prefix, *total the sum.
template <int NTH>
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned* wsum, unsigned* total) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[wp] = x;
  __syncthreads();
  unsigned before = 0, all = 0;
#pragma unroll
  for (int q = 0; q < NTH / 32; ++q) {
    before += q < wp ? wsum[q] : 0u;
    all += wsum[q];
  }
  __syncthreads();
  *total = all;
  return before + x - v;
}

// The block's wide droplets (sorted indices in list[0..nw)), one after another: the partners of
// the wide search are added to each droplet's count and its record is marked (scr = -1), so that
// the emit pass writes its pairs by wide_emit_block.
template <int NTH>
__device__ void wide_count_block(const unsigned* list, int nw, const double4* __restrict__ sp,
                                 const float4* __restrict__ spf, const unsigned* __restrict__ skey,
                                 const int* __restrict__ cs, int nc, double L, double cw, unsigned* __restrict__ cnt,
                                 int* __restrict__ scr, unsigned* wsum) {
  const float Lf = (float)L, hf = 0.5f * Lf, margin = (float)(1e-6 * L);
  for (int e = 0; e < nw; ++e) {
    const int s = (int)list[e];
    const double4 me = sp[s];
    const float4 mf = spf[s];
    const WideCell w = wide_cell(skey[s], nc, me.w, cw);
    const int items = w.ax * w.ax * w.ax;
    const int per = (items + NTH - 1) / NTH;
    unsigned c = 0;
    for (int it = threadIdx.x * per; it < items && it < (int)(threadIdx.x + 1) * per; ++it)
      c += wide_item<false>(it, false, s, w, me, mf, sp, spf, cs, nc, L, cw, Lf, hf, margin + 1e-6f * mf.w, nullptr,
                            0, 0);
    unsigned total;
    block_excl_scan<NTH>(c, wsum, &total);
    if (threadIdx.x == 0) {
      cnt[s] += total;
      scr[(long long)KEEP * s] = -1;
    }
  }
}

// All pairs of the block's wide droplets (neighbour search, then wide search) at off[s]...
template <int NTH>
__device__ void wide_emit_block(const unsigned* list, int nw, const double4* __restrict__ sp,
                                const float4* __restrict__ spf, const unsigned* __restrict__ skey,
                                const int* __restrict__ cs, int nc, double L, double cw,
                                const unsigned* __restrict__ off, int* __restrict__ pairs, long long cap,
                                unsigned* wsum) {
  const float Lf = (float)L, hf = 0.5f * Lf, margin = (float)(1e-6 * L);
  for (int e = 0; e < nw; ++e) {
    const int s = (int)list[e];
    const double4 me = sp[s];
    const float4 mf = spf[s];
    const float mar = margin + 1e-6f * mf.w;
    const WideCell w = wide_cell(skey[s], nc, me.w, cw);
    const int items = 14 + w.ax * w.ax * w.ax;
    const int per = (items + NTH - 1) / NTH;
    const int i0 = threadIdx.x * per, i1 = i0 + per < items ? i0 + per : items;
    unsigned c = 0;
    for (int it = i0; it < i1; ++it)
      c += wide_item<false>(it, true, s, w, me, mf, sp, spf, cs, nc, L, cw, Lf, hf, mar, nullptr, 0, 0);
    unsigned total;
    long long o = (long long)off[s] + block_excl_scan<NTH>(c, wsum, &total);
    for (int it = i0; it < i1; ++it)
      o += wide_item<true>(it, true, s, w, me, mf, sp, spf, cs, nc, L, cw, Lf, hf, mar, pairs, o, cap);
  }
}

template <int CT>  // threads per block: fewer for sparse columns (a multi-box collider's small boxes)
__global__ void __launch_bounds__(CT)
k_col_pairs(const double4* __restrict__ sp, const float4* __restrict__ spf, const unsigned* __restrict__ skey,
            const int* __restrict__ cs, int nc, int parts, double L, double cw, int cap_smem,
            unsigned* __restrict__ cnt, int* __restrict__ scr) {
  extern __shared__ __align__(16) unsigned char cp_smem[];
  float4* colbuf = reinterpret_cast<float4*>(cp_smem);
  int* cst = reinterpret_cast<int*>(cp_smem + sizeof(float4) * (size_t)cap_smem);  // 5 x (nc + 1) cell starts
  __shared__ long long kq[5];
  __shared__ int lo[5], so[6], dl[5];
  __shared__ float shx[5], shy[5];
  __shared__ unsigned wlist[CT], nwide, wsum[CT / 32];
  if (threadIdx.x == 0) nwide = 0u;
  const long long colg = blockIdx.x / parts;  // (box, cx, cy) of a multi-box collider
  const int part = (int)(blockIdx.x % parts);
  const long long ncol = (long long)nc * nc;
  const long long bbase = (colg / ncol) * ncol * nc;  // the box's first cell
  const long long col = colg % ncol;
  const int cx = (int)(col / nc), cy = (int)(col % nc);
  const float Lf = (float)L, margin = (float)(1e-6 * L);
  if (threadIdx.x < 5) {
    int ox, oy;
    col_offset(threadIdx.x, ox, oy);
    kq[threadIdx.x] = bbase + ((long long)((cx + ox) % nc) * nc + (cy + oy + nc) % nc) * nc;
    shx[threadIdx.x] = (cx + ox >= nc) ? -Lf : 0.f;
    shy[threadIdx.x] = (cy + oy >= nc) ? -Lf : ((cy + oy < 0) ? Lf : 0.f);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 5 * (nc + 1); e += CT) {
    const int q = e / (nc + 1), z = e - q * (nc + 1);
    cst[e] = cs[kq[q] + z];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int q = 0; q < 5; ++q) {
      lo[q] = cst[q * (nc + 1)];
      so[q] = acc;
      acc += cst[q * (nc + 1) + nc] - lo[q];
    }
    so[5] = acc;
  }
  __syncthreads();
  const bool staged = so[5] <= cap_smem;  // block-uniform
  if (threadIdx.x < 5) dl[threadIdx.x] = staged ? lo[threadIdx.x] - so[threadIdx.x] : 0;
  if (staged) {
    for (int q = 0; q < 5; ++q) {
      const int n_q = so[q + 1] - so[q];
      for (int t = threadIdx.x; t < n_q; t += CT) colbuf[so[q] + t] = spf[lo[q] + t];
    }
  }
  __syncthreads();
  const int len0 = so[1] - so[0];
  // rounds of CT droplets; after each, the block counts the round's wide droplets' partners
  // beyond the neighbour cells together
  for (int t0 = part * CT; t0 < len0; t0 += parts * CT) {
    const int t = t0 + threadIdx.x;
    if (t < len0) {
      const int i = lo[0] + t;
      const int cz = (int)(skey[i] - (unsigned)kq[0]);
      const bool wide =
          staged ? col_visit<true>(i, t, sp, spf, colbuf, cst, dl, shx, shy, cz, nc, L, cw, Lf, margin, cnt, scr)
                 : col_visit<false>(i, t, sp, spf, colbuf, cst, dl, shx, shy, cz, nc, L, cw, Lf, margin, cnt, scr);
      if (wide) wlist[atomicAdd(&nwide, 1u)] = (unsigned)i;
    }
    __syncthreads();
    const int nw = (int)nwide;  // block-uniform
    if (nw) wide_count_block<CT>(wlist, nw, sp, spf, skey, cs, nc, L, cw, cnt, scr, wsum);
    __syncthreads();
    if (threadIdx.x == 0) nwide = 0u;
    __syncthreads();
  }
}

// Pairs of sorted droplet i at off[i]..: copied from scr when it has at most KEEP partners,
// otherwise found again from global memory in the same visiting order.  The block takes rounds
// of EMIT_THREADS droplets; the round's wide droplets (scr marked by the column visit) are
// emitted by the whole block after the round (wide_emit_block).
constexpr int EMIT_THREADS = 256;

__global__ void __launch_bounds__(EMIT_THREADS)
k_emit_pairs(const double4* __restrict__ sp, const float4* __restrict__ spf, const unsigned* __restrict__ skey,
             const int* __restrict__ cs, int nc, double L, double cw, long long n, const unsigned* __restrict__ off,
             const int* __restrict__ scr, int* __restrict__ pairs, long long cap) {
  __shared__ unsigned wlist[EMIT_THREADS], nwide, wsum[EMIT_THREADS / 32];
  if (threadIdx.x == 0) nwide = 0u;
  __syncthreads();
  const float Lf = (float)L, hf = 0.5f * Lf, margin = (float)(1e-6 * L);
  for (long long base = (long long)blockIdx.x * EMIT_THREADS; base < n; base += (long long)gridDim.x * EMIT_THREADS) {
    const long long ii = base + threadIdx.x;
    const int i = (int)ii;
    const unsigned cnt = ii < n ? off[i + 1] - off[i] : 0u;
    if (cnt > 0 && scr[(long long)KEEP * i] < 0) {
      wlist[atomicAdd(&nwide, 1u)] = (unsigned)i;
    } else if (cnt > 0 && cnt <= (unsigned)KEEP) {
      const long long o0 = off[i];
      for (unsigned k = 0; k < cnt; ++k)
        if (o0 + k < cap) { pairs[2 * (o0 + k)] = i; pairs[2 * (o0 + k) + 1] = scr[(long long)KEEP * i + k]; }
    } else if (cnt > 0) {
      const unsigned key = skey[i];
      const unsigned nc3 = (unsigned)nc * nc * nc;
      const long long kb = (long long)(key / nc3) * nc3;  // the box's first cell
      const int cz = (int)(key % (unsigned)nc), cy = (int)((key / nc) % nc), cx = (int)((key / ((unsigned)nc * nc)) % nc);
      const float4 mf = spf[i];
      const float mar = margin + 1e-6f * mf.w;
      const double4 me = sp[i];
      long long o = off[i];
      for (int r = 0; r < 14; ++r) {
        int q, dz;
        if (r < 2) { q = 0; dz = r; }
        else { q = 1 + (r - 2) / 3; dz = (r - 2) % 3 - 1; }
        const int z = (cz + dz + nc) % nc;
        const int ox = q < 2 ? 0 : 1;
        const int oy = q == 0 ? 0 : (q == 1 ? 1 : q - 3);
        const long long k = kb + ((long long)((cx + ox) % nc) * nc + (cy + oy + nc) % nc) * nc + z;
        const int g1 = cs[k + 1];
        for (int g = r == 0 ? i + 1 : cs[k]; g < g1; ++g) {
          if (!near_f(mf, spf[g], Lf, hf, mar)) continue;
          if (!overlap_near(me, sp[g], L, cw)) continue;
          if (o < cap) { pairs[2 * o] = i; pairs[2 * o + 1] = g; }
          ++o;
        }
      }
    }
    __syncthreads();
    const int nw = (int)nwide;  // block-uniform
    if (nw) wide_emit_block<EMIT_THREADS>(wlist, nw, sp, spf, skey, cs, nc, L, cw, off, pairs, cap, wsum);
    __syncthreads();
    if (threadIdx.x == 0) nwide = 0u;
    __syncthreads();
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

// Pairs per box, sorted order (nc >= 3: the pairs of sorted droplet s are counted at off[s], and
// box b's droplets are the sorted slots start[b nc^3] .. start[(b + 1) nc^3] - 1).
__global__ void k_box_counts_sorted(const unsigned* __restrict__ off, const int* __restrict__ start, long long nc3,
                                    int nbox, int64_t* __restrict__ bc) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += gridDim.x * blockDim.x)
    bc[b] = (int64_t)off[start[(b + 1) * nc3]] - (int64_t)off[start[b * nc3]];
}

// Pairs per box, droplet order (nc < 3: counts are indexed by droplet); bc zeroed before.
__global__ void k_box_counts_ids(const unsigned* __restrict__ off, const int* __restrict__ box, long long n,
                                 int64_t* __restrict__ bc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned c = off[i + 1] - off[i];
    if (c) atomicAdd(reinterpret_cast<unsigned long long*>(bc + (box ? box[i] : 0)), (unsigned long long)c);
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
  int nbox = 1;  // boxes of a multi-box collider: cells (box, cx, cy, cz), box major
  unsigned *key = nullptr, *val = nullptr, *key2 = nullptr, *val2 = nullptr, *hist = nullptr, *cnt = nullptr;
  int* start = nullptr;  // cell starts, ncell + 1 entries
  double4* sp = nullptr;
  float4* spf = nullptr;
  int* scr = nullptr;  // first KEEP partners of each sorted droplet
  unsigned* status = nullptr;
  unsigned* nbig = nullptr;  // number of cells above kSmallCell droplets (counting sort)
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

int ld_collider_create(ld_collider** out, int64_t nmax, int32_t nc) { return ld_collider_create_boxes(out, nmax, nc, 1); }

int ld_collider_create_boxes(ld_collider** out, int64_t nmax, int32_t nc, int32_t nbox) {
  if (!out || nmax < 1 || nmax > (1LL << 31) - 2 || nc < 1 || nbox < 1 ||
      (long long)nc * nc * nc * nbox > (1LL << 31) - 2)
    return ld_fail(LD_ERR_ARG, "ld_collider_create: bad arguments");
  *out = nullptr;
  ld_collider* c = new (std::nothrow) ld_collider();
  if (!c) return ld_fail(LD_ERR_NOMEM, "host allocation failed");
  c->nmax = nmax;
  c->nc = nc;
  c->nbox = nbox;
  c->nblocks = (int)((nmax + RS_TILE - 1) / RS_TILE);
  const long long ncell = (long long)nc * nc * nc * nbox;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
  A((void**)&c->key, 4 * nmax);
  A((void**)&c->val, 4 * nmax);
  A((void**)&c->key2, 4 * nmax);
  A((void**)&c->val2, 4 * nmax);
  A((void**)&c->hist, 4 * (size_t)RADIX * c->nblocks);
  A((void**)&c->cnt, 4 * ((nmax > ncell ? nmax : ncell) + 1));
  A((void**)&c->start, 4 * (ncell + 1));
  A((void**)&c->sp, sizeof(double4) * nmax);
  A((void**)&c->spf, sizeof(float4) * nmax);
  A((void**)&c->scr, sizeof(int) * KEEP * nmax);
  A((void**)&c->status, sizeof(unsigned));
  A((void**)&c->nbig, sizeof(unsigned));
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
  cudaFree(c->cnt); cudaFree(c->start); cudaFree(c->sp); cudaFree(c->spf); cudaFree(c->scr); cudaFree(c->status);
  cudaFree(c->nbig);
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
  if (c && c->nbox != 1) return ld_fail(LD_ERR_ARG, "ld_collide: a multi-box collider needs ld_collide_boxes");
  return ld_collide_boxes(c, pos, radius, nullptr, n, L, pairs, cap, count, nullptr, stream);
}

int ld_collide_boxes(ld_collider* c, const double* pos, const double* radius, const int32_t* box, int64_t n, double L,
                     int32_t* pairs, int64_t cap, int64_t* count, int64_t* box_counts, void* stream) {
  if (!c || !count || n < 0 || n > c->nmax || cap < 0 || !(L > 0) || (n > 0 && (!pos || !radius)) ||
      (n > 0 && cap > 0 && !pairs) || (c->nbox > 1 && n > 0 && !box))
    return ld_fail(LD_ERR_ARG, "ld_collide: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = c->nc;
  const double cw = L / nc;
  const long long nc3 = (long long)nc * nc * nc;
  const long long ncell = nc3 * c->nbox;
  if (box_counts) LD_CUDA_CHECK(cudaMemsetAsync(box_counts, 0, sizeof(int64_t) * c->nbox, s));
  if (n == 0) {
    LD_CUDA_CHECK(cudaMemsetAsync(count, 0, sizeof(int64_t), s));
    return LD_OK;
  }
  {
    ProfScope ps(c->trace, KID_COLL_SORT, s);
    if (ncell + 1 > (long long)SCAN_TILE * SCAN_TILE) {
      // more cells than one scan handles: stable radix sort of the keys, starts by binary search
      k_cell_keys<<<gridn(n, 256), 256, 0, s>>>(pos, n, L, cw, nc, c->key, c->val, box);
      int bits = 1;
      while ((1LL << bits) < ncell) ++bits;
      if (int rc = ld_radix_sort_u32(c, c->key, c->val, n, bits, stream)) return rc;
      k_cell_starts<<<gridn(ncell + 1, 256), 256, 0, s>>>(c->key, n, ncell, c->start);
      k_sorted_copy<<<gridn(n, 256), 256, 0, s>>>(pos, radius, c->val, n, L, c->sp, c->spf);
    } else {
      // counting sort by cell (the same order): keys (c->key2) and arrival ranks (c->val2),
      // occupancies -> starts in c->start, unordered runs scattered into c->cnt, then every
      // droplet placed by its rank within its cell into c->val with the sorted keys (c->key) and
      // copies (cells above kSmallCell: listed in c->val2, sorted by k_cell_big)
      unsigned* occ = reinterpret_cast<unsigned*>(c->start);
      LD_CUDA_CHECK(cudaMemsetAsync(occ, 0, sizeof(unsigned) * (size_t)(ncell + 1), s));
      LD_CUDA_CHECK(cudaMemsetAsync(c->nbig, 0, sizeof(unsigned), s));
      k_cell_count<<<gridn(n, 256), 256, 0, s>>>(pos, n, L, cw, nc, c->key2, c->val2, occ, box);
      if (int rc = scan_u32(c, occ, ncell + 1, s)) return rc;
      k_cell_scatter<<<gridn(n, 256), 256, 0, s>>>(c->key2, c->val2, c->start, n, c->cnt);
      k_cell_place<<<gridn(n, 256), 256, 0, s>>>(c->key2, c->start, c->cnt, n, pos, radius, L, c->val, c->key, c->sp,
                                                 c->spf, c->val2, c->nbig);
      k_cell_big<<<148, 512, 0, s>>>(c->start, c->val2, c->nbig, c->cnt, pos, radius, L, c->val, c->key, c->sp,
                                     c->spf);
    }
  }
  ProfScope ps(c->trace, KID_COLL_PAIRS, s);
  LD_CUDA_CHECK(cudaMemsetAsync(c->cnt + n, 0, 4, s));
  if (nc >= 3) {
    // block per cell column (and part); pairs come out as sorted-array indices and are mapped
    // back to droplet indices by k_map_pairs
    const long long ncol = (long long)nc * nc * c->nbox;  // cell columns of every box
    const long long per_col = (n + ncol - 1) / ncol;
    const long long parts = per_col > 512 ? (per_col + 511) / 512 : 1;
    const size_t starts_bytes = sizeof(int) * 5 * (size_t)(nc + 1);
    if (ncol * parts > 0x7fffffffLL || starts_bytes > 64 * 1024)
      return ld_fail(LD_ERR_UNSUPPORTED, "ld_collide: too many cells per side (%d)", nc);
    long long want = 5 * per_col + (5 * per_col) / 4 + 256;  // typical staged rows, with headroom
    const long long room = (long long)((220 * 1024 - starts_bytes) / sizeof(float4));
    if (want > kColSmemRows) want = kColSmemRows;
    if (want > room) want = room;
    const int cap_smem = (int)want;
    const size_t smem = sizeof(float4) * (size_t)cap_smem + starts_bytes;
    // blocks of 64, 128 or 192 threads where columns hold few droplets (the boxes of an ensemble;
    // about 150 per column at 1e6 droplets in 82^3 cells), 256 otherwise: threads without a
    // droplet would only wait at the block's barriers
    if (per_col <= 64) {
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_col_pairs<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_col_pairs<64><<<(unsigned)(ncol * parts), 64, smem, s>>>(c->sp, c->spf, c->key, c->start, nc, (int)parts, L,
                                                                 cw, cap_smem, c->cnt, c->scr);
    } else if (per_col <= 128) {
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_col_pairs<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_col_pairs<128><<<(unsigned)(ncol * parts), 128, smem, s>>>(c->sp, c->spf, c->key, c->start, nc, (int)parts, L,
                                                                   cw, cap_smem, c->cnt, c->scr);
    } else if (per_col <= 192) {
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_col_pairs<192>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      // shared memory, not registers, would otherwise hold it to 5 blocks per SM
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_col_pairs<192>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      k_col_pairs<192><<<(unsigned)(ncol * parts), 192, smem, s>>>(c->sp, c->spf, c->key, c->start, nc, (int)parts, L,
                                                                   cw, cap_smem, c->cnt, c->scr);
    } else {
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_col_pairs<COL_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
      k_col_pairs<COL_THREADS><<<(unsigned)(ncol * parts), COL_THREADS, smem, s>>>(
          c->sp, c->spf, c->key, c->start, nc, (int)parts, L, cw, cap_smem, c->cnt, c->scr);
    }
    if (int rc = scan_u32(c, c->cnt, n + 1, s)) return rc;
    k_emit_pairs<<<gridn(n, EMIT_THREADS), EMIT_THREADS, 0, s>>>(c->sp, c->spf, c->key, c->start, nc, L, cw, n,
                                                                 c->cnt, c->scr, pairs, cap);
    k_map_pairs<<<gridn(cap, 256), 256, 0, s>>>(c->cnt + n, cap, c->val, pairs);
    if (box_counts)
      k_box_counts_sorted<<<(c->nbox + 255) / 256, 256, 0, s>>>(c->cnt, c->start, nc3, c->nbox, box_counts);
  } else {
    const int* end = c->start + 1;  // end of cell k = start of cell k + 1
    k_pairs<0, true><<<gridn(n, 128), 128, 0, s>>>(c->sp, c->val, c->key, c->start, end, n, nc, L, c->cnt,
                                                   nullptr, nullptr, 0);
    if (int rc = scan_u32(c, c->cnt, n + 1, s)) return rc;
    k_pairs<1, true><<<gridn(n, 128), 128, 0, s>>>(c->sp, c->val, c->key, c->start, end, n, nc, L, nullptr,
                                                   c->cnt, pairs, cap);
    if (box_counts) k_box_counts_ids<<<gridn(n, 256), 256, 0, s>>>(c->cnt, box, n, box_counts);
  }
  k_finish<<<1, 1, 0, s>>>(c->cnt, n, cap, count, c->status);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_cell_order(ld_collider* c, const double* pos, int64_t n, double L, uint32_t* order, void* stream) {
  if (c && c->nbox != 1) return ld_fail(LD_ERR_ARG, "ld_cell_order: a multi-box collider needs ld_cell_order_boxes");
  return ld_cell_order_boxes(c, pos, nullptr, n, L, order, stream);
}

int ld_cell_order_boxes(ld_collider* c, const double* pos, const int32_t* box, int64_t n, double L, uint32_t* order,
                        void* stream) {
  if (!c || n < 0 || n > c->nmax || !(L > 0) || (n > 0 && (!pos || !order)) || (c->nbox > 1 && n > 0 && !box))
    return ld_fail(LD_ERR_ARG, "ld_cell_order: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  ProfScope ps(c->trace, KID_CELL_ORDER, s);
  const int nc = c->nc;
  const long long ncell = (long long)nc * nc * nc * c->nbox;
  k_cell_keys<<<gridn(n, 256), 256, 0, s>>>(pos, n, L, L / nc, nc, c->key, c->val, box);
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

int ld_copy_async(void* dst, const void* src, int64_t bytes, void* stream) {
  if (bytes < 0 || (bytes > 0 && (!dst || !src))) return ld_fail(LD_ERR_ARG, "ld_copy_async: bad arguments");
  if (bytes == 0) return LD_OK;
  LD_CUDA_CHECK(cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
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
