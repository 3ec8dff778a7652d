// Learned interpolation: an MLP that predicts the correction from tricubic interpolation to the
// exact spectral velocity at a droplet, from the droplet's 4x4x4 stencil of (u, v, w) and its
// fractional cell offset.  No counterpart in the reference.
//
// Network: 195 inputs -> 128 SiLU -> 128 SiLU -> 3.  Operands are BF16 on the tensor cores
// (tcgen05.mma, FP32 accumulators in tensor memory), for inference and training alike; master
// weights, biases and the optimiser are FP32.
//
// Features of a point with stencil values s (192 = 3 components x 64 taps, tap order
// c*64 + a*16 + b*4 + q for offsets a, b, q in -1..2 along x, y, z) and cell offsets t (3):
//   D_c      = (P x P x P) s_c    per component: the discrete polynomial basis of orders 0..3
//              on 4 points along each axis, rows (1,1,1,1), (-3,-1,1,3), (1,-1,-1,1), (-1,3,-3,1)
//              (orthogonal; their norms are absorbed by the feature scales) (FP32)
//   scale    = RMS of all 192 coefficients (scale mode 0), or of the 162 coefficients of total
//              order >= 3 (mode 1: tracks the small-scale content the correction depends on,
//              so the normalised targets drift less while a flow develops), + 1e-30, both in
//              the basis above
//   x[0:192] = D / scale * fs,  x[192:195] = t - 0.5,  x[195:208] = 0     (canonical frame)
//   u(point) = tricubic(s, t) + scale * os * MLP(x)                     (back in the grid frame)
// Canonical frame: the exact correction is equivariant under the 48 reflections and axis
// permutations of the cube, and the flow is statistically isotropic.  Each axis whose offset
// exceeds 1/2 is reflected (offset -> 1 - offset, that velocity component and the odd-order
// coefficients along it change sign), then the axes are ordered by decreasing reflected offset
// (stable).  Features, targets and outputs are expressed in that frame, which shrinks the input
// domain 48-fold.
// The correction lives in the high-order coefficients, which are 1e-2..1e-4 of the values: the
// transform happens in FP32 before the BF16 rounding, and the per-coefficient feature scales fs
// (64, shared by the components) bring every feature to O(1).  fs and the output scale os are
// set from sample statistics before training and are not trained.  Per-point normalisation makes
// the prediction scale with the field, as the exact correction (a linear functional of the
// field) does.
//
// Parameter vector (FP32, contiguous), "params":
//   W1 [208][128] (input-major; rows 195..207 stay zero)  b1 [128]
//   W2 [128][128]                                          b2 [128]
//   W3 [128][8]   (columns 3..7 stay zero)                 b3 [8]
//   fs [64]       os [8] (os[0]: output scale, os[1]: scale mode)
// Packed BF16 copies for the tensor cores ("packed"), output-major with padded rows:
//   W1t [128][KP1]   W2t [128][KP2]   W2n [128][KP2] (= W2, input-major)   W3t [8][KP2]   W3n [128][8]
//   then W1t, W2t and W3t (16 rows) once more in the tensor-core tile layout (tile_elem), which the
//   training kernel copies to shared memory as three bulk copies
#include <cmath>

#include <cuda_bf16.h>

#include "ld_internal.cuh"
#include "ld_kernels.cuh"

namespace {

using namespace ld;

constexpr int D_IN = 195, K1 = 208, H = 128, D_OUT = 3, N3 = 8;
constexpr int KP1 = 216;  // padded row stride (bf16) of the packed 208-long rows
constexpr int KP2 = 136;  // padded row stride of the packed 128-long rows

constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + K1 * H;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H * N3;
constexpr int OFF_FS = OFF_B3 + N3;
constexpr int OFF_OS = OFF_FS + 64;
constexpr int N_PARAMS = OFF_OS + 8;

constexpr int P_W1T = 0;
constexpr int P_W2T = P_W1T + H * KP1;
constexpr int P_W2N = P_W2T + H * KP2;
constexpr int P_W3T = P_W2N + H * KP2;
constexpr int P_W3N = P_W3T + N3 * KP2;
constexpr int N3P = 16;                     // layer-3 N padded for M = 128
constexpr int P_TW1 = P_W3N + H * N3;       // W1 in the tensor-core tile layout (rows o, K = k)
constexpr int P_TW2 = P_TW1 + H * K1;       // W2 in the tile layout (rows o, K = i)
constexpr int P_TW3 = P_TW2 + H * H;        // W3 in the tile layout (16 rows c, K = i; rows 3..15 zero)
constexpr int N_PACKED = P_TW3 + N3P * H;
static_assert((P_TW1 * 2) % 16 == 0 && (P_TW2 * 2) % 16 == 0 && (P_TW3 * 2) % 16 == 0, "bulk-copy alignment");

// Element index of (row, k) in the tensor-core tile layout of a K-major operand with `rows` rows:
// 8x8 core matrices (8 rows of 8 consecutive k, 128 contiguous bytes), K-chunk major.
__host__ __device__ constexpr int tile_elem(int row, int k, int rows) {
  return ((k / 8) * (rows / 8) + row / 8) * 64 + (row % 8) * 8 + k % 8;
}

using bf16 = __nv_bfloat16;

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}

// SiLU with the logistic function from the hardware tanh approximation, sigma(z) = (1 + tanh(z/2))/2
// (relative error ~5e-4, below the BF16 rounding of the activations); training and inference use
// the same function.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigm(float z) { return fmaf(0.5f, tanh_fast(0.5f * z), 0.5f); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigm(z);
  return s * (1.f + z * (1.f - s));
}

// ---- features of one point ------------------------------------------------------------------------
// The building blocks below are shared by the thread-per-sample training-sample kernel and the
// warp-cooperative inference kernel; every element goes through the same arithmetic in both,
// so training and inference features agree bit for bit.

// Discrete polynomial basis on 4 points (orders 0..3, rows (1,1,1,1), (-3,-1,1,3), (1,-1,-1,1),
// (-1,3,-3,1): orthogonal, not normalised; the feature scales absorb the norms), in place.
__device__ __forceinline__ void poly4(float* v, int stride) {
  const float s0 = v[0], s1 = v[stride], s2 = v[2 * stride], s3 = v[3 * stride];
  const float a = s0 + s3, b = s1 + s2, c = s3 - s0, d = s2 - s1;
  v[0] = a + b;
  v[stride] = fmaf(3.f, c, d);
  v[2 * stride] = a - b;
  v[3 * stride] = fmaf(-3.f, d, c);
}

// Frame code: bits 0-5 hold p[0..2] (canonical axis k <- grid axis p[k], 2 bits each), bits 6-8
// the reflection of grid axes 0..2.
__device__ __forceinline__ int frame_perm(int code, int k) { return (code >> (2 * k)) & 3; }
__device__ __forceinline__ float frame_sign(int code, int d) { return (code >> (6 + d)) & 1 ? -1.f : 1.f; }

__device__ __forceinline__ int make_frame(const float* toff, float* tc) {
  float r[3];
  int code = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const bool rf = toff[d] > 0.5f;
    r[d] = rf ? 1.f - toff[d] : toff[d];
    code |= (rf ? 1 : 0) << (6 + d);
  }
  // sort the offsets descending, carrying their axes (values move with the indices, so nothing
  // is indexed at run time)
  int p0 = 0, p1 = 1, p2 = 2, x;
  float a = r[0], b = r[1], c = r[2], y;
  if (b > a) { x = p0; p0 = p1; p1 = x; y = a; a = b; b = y; }
  if (c > b) { x = p1; p1 = p2; p2 = x; y = b; b = c; c = y; }
  if (b > a) { x = p0; p0 = p1; p1 = x; y = a; a = b; b = y; }
  tc[0] = a;
  tc[1] = b;
  tc[2] = c;
  return code | p0 | (p1 << 2) | (p2 << 4);
}

// Cell and canonical frame of a point: grid cell i (periodic), offsets t in grid units.
struct PtFrame {
  int i[3];
  int code;
  float tc[3];
};

__device__ __forceinline__ void point_frame(double px, double py, double pz, int N, double L, PtFrame& f) {
  const double sc = double(N) / L;
  const double q[3] = {px * sc, py * sc, pz * sc};
  float toff[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double fl = floor(q[d]);
    toff[d] = float(q[d] - fl);
    f.i[d] = int((long long)fl & (long long)(N - 1));  // periodic cell; N is a power of two
  }
  f.code = make_frame(toff, f.tc);
}

// Tricubic weights of the canonical offsets in the polynomial basis (per canonical axis): with
// U the basis above (row norms^2 4, 20, 4, 20), w.s = sum_i (U w)_i (U s)_i / |U_i|^2, so the
// tricubic value is sum_i D_i wh0[i0] wh1[i1] wh2[i2] with wh = (U w) / |U|^2.
__device__ __forceinline__ void tric_weight_axis(float t, float (&w)[4]) {
  w[0] = -t * (t - 1.f) * (t - 2.f) / 6.f;
  w[1] = (t + 1.f) * (t - 1.f) * (t - 2.f) / 2.f;
  w[2] = -(t + 1.f) * t * (t - 2.f) / 2.f;
  w[3] = (t + 1.f) * t * (t - 1.f) / 6.f;
  poly4(w, 1);
  w[0] *= 0.25f;
  w[1] *= 0.05f;
  w[2] *= 0.25f;
  w[3] *= 0.05f;
}
__device__ __forceinline__ void tric_weights(const float* tc, float (&wh)[3][4]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) tric_weight_axis(tc[k], wh[k]);
}

// A component's 64 taps live as 32 packed FP32 pairs: pair i holds tap i (canonical index
// j0 j1 j2 with j0 < 2) in .x and tap i + 32 (j0 + 2) in .y.  Along axes 2 and 1 the lines of j0
// and j0 + 2 are transformed together by packed instructions (__fadd2_rn / __ffma2_rn: each half
// rounds exactly as the scalar operation), along axis 0 the four taps of a line sit in two pairs
// and are transformed as scalars; every tap goes through exactly the operations of the scalar
// transform, so the coefficients are bit-identical to it.
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ void poly4x2(float2* v, int stride) {
  const float2 s0 = v[0], s1 = v[stride], s2 = v[2 * stride], s3 = v[3 * stride];
  const float2 a = __fadd2_rn(s0, s3), b = __fadd2_rn(s1, s2), c = __fadd2_rn(s3, neg2(s0)), d = __fadd2_rn(s2, neg2(s1));
  v[0] = __fadd2_rn(a, b);
  v[stride] = __ffma2_rn(make_float2(3.f, 3.f), c, d);
  v[2 * stride] = __fadd2_rn(a, neg2(b));
  v[3 * stride] = __ffma2_rn(make_float2(-3.f, -3.f), d, c);
}
// tap j of the packed layout
__device__ __forceinline__ float tap(const float2 (&v)[32], int j) { return j < 32 ? v[j].x : v[j - 32].y; }
__device__ __forceinline__ void set_tap(float2 (&v)[32], int j, float x) {
  if (j < 32) v[j].x = x;
  else v[j - 32].y = x;
}

// One component's 64 taps (canonical order, in registers) -> its polynomial coefficients, then
// the component's partial sums: squares, squares of total order >= 3, and its tricubic value.
// The three components are combined as (c0 + c1) + c2 by every caller, so all paths round
// identically; all indices are compile-time constants.
__device__ __forceinline__ void comp_transform(float2 (&v)[32]) {
#pragma unroll
  for (int a = 0; a < 8; ++a) poly4x2(v + 4 * a, 1);                         // along axis 2
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) poly4x2(v + 16 * a + q, 4);                  // along axis 1
#pragma unroll
  for (int e = 0; e < 16; ++e) {                                             // along axis 0
    float w4[4] = {v[e].x, v[e + 16].x, v[e].y, v[e + 16].y};
    poly4(w4, 1);
    v[e].x = w4[0];
    v[e + 16].x = w4[1];
    v[e].y = w4[2];
    v[e + 16].y = w4[3];
  }
}

struct CompSums {
  float ss, sh, tr;
};

// need_ss: also the sum of all squares (scale mode 0); mode 1 needs only sh.
__device__ __forceinline__ CompSums comp_sums(const float2 (&v)[32], const float (&wh)[3][4], bool need_ss = true) {
  CompSums p{0.f, 0.f, 0.f};
  if (need_ss) {
#pragma unroll
    for (int j = 0; j < 64; ++j) p.ss = fmaf(tap(v, j), tap(v, j), p.ss);
  }
#pragma unroll
  for (int j = 0; j < 64; ++j)
    if ((j >> 4) + ((j >> 2) & 3) + (j & 3) >= 3) p.sh = fmaf(tap(v, j), tap(v, j), p.sh);
  // tricubic value by separable contraction: z, then y, then x
  float t1[16];
#pragma unroll
  for (int q = 0; q < 16; ++q)
    t1[q] = fmaf(wh[2][3], tap(v, 4 * q + 3), fmaf(wh[2][2], tap(v, 4 * q + 2),
                 fmaf(wh[2][1], tap(v, 4 * q + 1), wh[2][0] * tap(v, 4 * q))));
  float tr = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const float t2 = fmaf(wh[1][3], t1[4 * a + 3], fmaf(wh[1][2], t1[4 * a + 2], fmaf(wh[1][1], t1[4 * a + 1], wh[1][0] * t1[4 * a])));
    tr = fmaf(wh[0][a], t2, tr);
  }
  p.tr = tr;
  return p;
}

__device__ __forceinline__ float scale_of(float ss0, float ss1, float ss2, float sh0, float sh1, float sh2,
                                          float mode) {
  const float ss = (ss0 + ss1) + ss2, sh = (sh0 + sh1) + sh2;
  return (mode != 0.f ? sqrtf(sh / 162.f) : sqrtf(ss / 192.f)) + 1e-30f;
}

// The 64 features of one component as 32 packed bf16 pairs: feature j = (tap j * inv) * fs[j],
// the two products of a pair of taps (j, j + 32) as packed instructions.  fs2[i] = (fs[i], fs[i + 32]).
__device__ __forceinline__ void comp_features(const float2 (&v)[32], const float2* fs2, float inv, unsigned (&w)[32]) {
  float2 x[32];
  const float2 inv2 = make_float2(inv, inv);
#pragma unroll
  for (int i = 0; i < 32; ++i) x[i] = __fmul2_rn(__fmul2_rn(v[i], inv2), fs2[i]);
#pragma unroll
  for (int j = 0; j < 32; ++j) w[j] = pack2(tap(x, 2 * j), tap(x, 2 * j + 1));
}

// The offset part of a row (columns 192..207): t - 1/2 for the three canonical offsets, zeros.
__device__ __forceinline__ void tail_features(const float* tc, unsigned (&w)[8]) {
  w[0] = pack2(tc[0] - 0.5f, tc[1] - 0.5f);
  w[1] = pack2(tc[2] - 0.5f, 0.f);
#pragma unroll
  for (int j = 2; j < 8; ++j) w[j] = 0u;
}

// Grid-memory offset, in scalar elements of the interleaved field (4 per grid point), of canonical
// index j along canonical axis k of a point (cell ci, frame code): along grid axis p[k], reversed
// when that axis is reflected.  Unsigned 32-bit: 4 N^3 <= 2^32 for N <= 1024.
__device__ __forceinline__ unsigned canon_offset(const int* ci, int code, int N, int k, int j) {
  const int d = frame_perm(code, k);
  const int o = (code >> (6 + d)) & 1 ? 3 - j : j;
  const int cid = d == 0 ? ci[0] : (d == 1 ? ci[1] : ci[2]);
  const unsigned g = (unsigned)((cid - 1 + o + N) & (N - 1));
  const unsigned n = (unsigned)N;
  return 4u * (d == 0 ? g * n * n : (d == 1 ? g * n : g));
}

// Canonical component c of the point's 64-tap stencil, straight from the interleaved field into
// registers (canonical tap order j0*16 + j1*4 + j2), without the frame's sign of the component,
// which is returned: the transform and the sums are odd or even in the sign and round
// symmetrically, so callers apply it exactly where it matters (features, canonical tricubic).
template <typename T>
__device__ __forceinline__ float gather_component(const vec4<T>* __restrict__ u4, int N, const PtFrame& f, int c,
                                                  float2 (&v)[32]) {
  const int d = frame_perm(f.code, c);
  const float sg = frame_sign(f.code, d);
  unsigned o0[4], o1[4], o2[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    o0[j] = canon_offset(f.i, f.code, N, 0, j) + (unsigned)d;  // the component folded in once
    o1[j] = canon_offset(f.i, f.code, N, 1, j);
    o2[j] = canon_offset(f.i, f.code, N, 2, j);
  }
  // one warp-uniform base pointer and a 32-bit offset per tap
  const T* base = reinterpret_cast<const T*>(u4);
#pragma unroll
  for (int j0 = 0; j0 < 4; ++j0)
#pragma unroll
    for (int j1 = 0; j1 < 4; ++j1) {
      const unsigned o01 = o0[j0] + o1[j1];
#pragma unroll
      for (int j2 = 0; j2 < 4; ++j2) set_tap(v, 16 * j0 + 4 * j1 + j2, float(__ldg(base + (o01 + o2[j2]))));
    }
  return sg;
}

// The same gather from the point's canonical offsets o[k][j] (canon_offset of axis k, index j),
// computed elsewhere.
template <typename T>
__device__ __forceinline__ float gather_component_at(const vec4<T>* __restrict__ u4, const PtFrame& f, int c,
                                                     const unsigned (&o)[3][4], float2 (&v)[32]) {
  const int d = frame_perm(f.code, c);
  const float sg = frame_sign(f.code, d);
  const T* base = reinterpret_cast<const T*>(u4);
#pragma unroll
  for (int j0 = 0; j0 < 4; ++j0)
#pragma unroll
    for (int j1 = 0; j1 < 4; ++j1) {
      const unsigned o01 = o[0][j0] + (unsigned)d + o[1][j1];
#pragma unroll
      for (int j2 = 0; j2 < 4; ++j2) set_tap(v, 16 * j0 + 4 * j1 + j2, float(__ldg(base + (o01 + o[2][j2]))));
    }
  return sg;
}

// Thread-per-point features (training samples): st is a 192-float scratch.  Returns the scale;
// tric (grid frame), the canonical tricubic value and the frame code come back through the
// arguments.
template <typename T>
__device__ __forceinline__ float point_features(const vec4<T>* __restrict__ u4, int N, double L, double px, double py,
                                                double pz, const float* __restrict__ params, float* st, bf16* row,
                                                float* tric_grid, int& code, float* tric_can) {
  PtFrame f;
  point_frame(px, py, pz, N, L, f);
  float wh[3][4];
  tric_weights(f.tc, wh);
  CompSums cs[3];
  float sgc[3];
  for (int c = 0; c < 3; ++c) {
    float2 v[32];
    sgc[c] = gather_component<T>(u4, N, f, c, v);
    comp_transform(v);
    cs[c] = comp_sums(v, wh);
#pragma unroll
    for (int j = 0; j < 64; ++j) st[64 * c + j] = tap(v, j);
  }
  const float scale = scale_of(cs[0].ss, cs[1].ss, cs[2].ss, cs[0].sh, cs[1].sh, cs[2].sh, params[OFF_OS + 1]);
  const float inv = 1.f / scale;
  const float* fs = params + OFF_FS;
  float2 fs2[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) fs2[i] = make_float2(fs[i], fs[i + 32]);
  unsigned* rw = reinterpret_cast<unsigned*>(row);
  for (int c = 0; c < 3; ++c) {
    float2 v[32];
#pragma unroll
    for (int j = 0; j < 64; ++j) set_tap(v, j, st[64 * c + j]);
    unsigned w[32];
    comp_features(v, fs2, sgc[c] * inv, w);
#pragma unroll
    for (int j = 0; j < 32; ++j) rw[32 * c + j] = w[j];
  }
  unsigned wt[8];
  tail_features(f.tc, wt);
#pragma unroll
  for (int j = 0; j < 8; ++j) rw[96 + j] = wt[j];
  code = f.code;
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    tric_can[cc] = sgc[cc] * cs[cc].tr;  // cs.tr is the unsigned (grid-frame) value
    tric_grid[frame_perm(code, cc)] = cs[cc].tr;
  }
  return scale;
}

// ---- packing -----------------------------------------------------------------------------------
__global__ void k_mlp_pack(const float* __restrict__ p, bf16* __restrict__ q) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N_PACKED; e += gridDim.x * blockDim.x) {
    float v = 0.f;
    if (e < P_W2T) {  // W1t[o][k] = W1[k][o]
      const int o = (e - P_W1T) / KP1, k = (e - P_W1T) % KP1;
      v = k < K1 ? p[OFF_W1 + k * H + o] : 0.f;
    } else if (e < P_W2N) {  // W2t[o][i] = W2[i][o]
      const int o = (e - P_W2T) / KP2, i = (e - P_W2T) % KP2;
      v = i < H ? p[OFF_W2 + i * H + o] : 0.f;
    } else if (e < P_W3T) {  // W2n[i][o] = W2[i][o]
      const int i = (e - P_W2N) / KP2, o = (e - P_W2N) % KP2;
      v = o < H ? p[OFF_W2 + i * H + o] : 0.f;
    } else if (e < P_W3N) {  // W3t[o][i] = W3[i][o]
      const int o = (e - P_W3T) / KP2, i = (e - P_W3T) % KP2;
      v = i < H ? p[OFF_W3 + i * N3 + o] : 0.f;
    } else if (e < P_TW1) {  // W3n[i][o] = W3[i][o]
      const int r = e - P_W3N;
      v = p[OFF_W3 + r];
    } else {  // the tile copies: element t of a tile with `rows` rows holds (row, k)
      const bool w1 = e < P_TW2, w2 = !w1 && e < P_TW3;
      const int t = e - (w1 ? P_TW1 : (w2 ? P_TW2 : P_TW3));
      const int rows = w1 || w2 ? H : N3P;
      const int cm = t / 64, w = t % 64;
      const int row = (cm % (rows / 8)) * 8 + w / 8, k = (cm / (rows / 8)) * 8 + w % 8;
      if (w1) v = p[OFF_W1 + k * H + row];
      else if (w2) v = p[OFF_W2 + k * H + row];
      else v = row < N3 ? p[OFF_W3 + k * N3 + row] : 0.f;
    }
    q[e] = __float2bfloat16_rn(v);
  }
}

// ---- inference, in two kernels ------------------------------------------------------------------
// k_mlp_features writes each droplet's feature row (bf16, K1 columns) to global memory in the
// tensor-core tile layout (tiles of TM rows, 8x8 core matrices, see blk_off) and its aux
// (tricubic xyz in the grid frame, scale, frame code) as 8 floats; k_mlp_forward_tc runs the
// three layers on the tensor cores and writes the velocities.
// Tensor-core tile layout of a K-major bf16 operand with `rows` rows: 8x8 core matrices (8 rows of
// 16 bytes, 128 contiguous bytes), K-chunk major: byte offset of (row, 8-element K chunk kc).
__host__ __device__ constexpr int blk_off(int row, int kc, int rows) {
  return (kc * (rows / 8) + row / 8) * 128 + (row % 8) * 16;
}
constexpr int TM = 128;                             // droplets per tensor-core tile
constexpr int TILE_X_BYTES = TM * K1 * 2;           // one tile of feature rows

// k_mlp_features: lane 3r + c of a warp takes canonical component c of droplet r (10 droplets
// per warp; lanes 30, 31 shadow droplet 9): the component's stencil is gathered into registers,
// transformed, reduced to its partial sums, and the three lanes of a droplet combine them by
// shuffles; each lane writes its 64 features (128 contiguous bytes of the tile layout), lane 3r
// also the offsets and the aux (tricubic xyz in the grid frame, scale, frame code).
constexpr int FDROP = 10;
constexpr int FTHREADS = 256;

template <typename T>
__global__ void __launch_bounds__(FTHREADS, 2)
k_mlp_features(const vec4<T>* __restrict__ u4, int N, double L, const double* __restrict__ pos, long long n,
               const float* __restrict__ params, bf16* __restrict__ Xg, float* __restrict__ auxg) {
  const int lane = threadIdx.x & 31;
  const int r = lane < 3 * FDROP ? lane / 3 : FDROP - 1;
  const int c = lane < 3 * FDROP ? lane - 3 * r : 0;
  __shared__ __align__(16) float2 fs2[32];  // feature scales as pairs (fs[i], fs[i + 32]), warp-uniform reads
  if (threadIdx.x < 32) fs2[threadIdx.x] = make_float2(params[OFF_FS + threadIdx.x], params[OFF_FS + 32 + threadIdx.x]);
  __syncthreads();
  const float mode = params[OFF_OS + 1];
  const long long ngroups = (n + FDROP - 1) / FDROP;
  // each CTA takes a contiguous range of groups (its warps interleaved inside it): CTAs run in
  // launch order, so the resident ones work on one contiguous window of the (cell-sorted)
  // droplets and the field lines their stencils share stay in L2
  constexpr int WPB = FTHREADS / 32;
  const long long per = (ngroups + gridDim.x - 1) / gridDim.x;
  const long long g_lo = (long long)blockIdx.x * per;
  const long long g_hi = g_lo + per < ngroups ? g_lo + per : ngroups;
  const long long wg = g_lo + (threadIdx.x >> 5);
  constexpr long long nw = WPB;
  // positions of the warp's next group are loaded while the current one is processed
  double px = 0.0, py = 0.0, pz = 0.0;
  if (wg < g_hi) {
    const long long i0 = wg * FDROP + r, ii0 = i0 < n ? i0 : n - 1;
    px = pos[3 * ii0]; py = pos[3 * ii0 + 1]; pz = pos[3 * ii0 + 2];
  }
  for (long long grp = wg; grp < g_hi; grp += nw) {
    const long long i = grp * FDROP + r;
    PtFrame f;
    point_frame(px, py, pz, N, L, f);
    if (grp + nw < g_hi) {
      const long long i1 = (grp + nw) * FDROP + r, ii1 = i1 < n ? i1 : n - 1;
      px = pos[3 * ii1]; py = pos[3 * ii1 + 1]; pz = pos[3 * ii1 + 2];
    }
    // the three lanes of a droplet split the per-point work by canonical axis (lane 3r + c takes
    // axis c's stencil offsets and tricubic weights) and exchange it by shuffles
    const int b0 = 3 * r;
    unsigned o[3][4];
    float wh[3][4];
    {
      unsigned oc[4];
      float wc[4];
      const float tcc = c == 0 ? f.tc[0] : (c == 1 ? f.tc[1] : f.tc[2]);
#pragma unroll
      for (int j = 0; j < 4; ++j) oc[j] = canon_offset(f.i, f.code, N, c, j);
      tric_weight_axis(tcc, wc);
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          o[k][j] = __shfl_sync(0xffffffffu, oc[j], b0 + k);
          wh[k][j] = __shfl_sync(0xffffffffu, wc[j], b0 + k);
        }
    }
    float2 v[32];
    const float sg = gather_component_at<T>(u4, f, c, o, v);
    comp_transform(v);
    const CompSums cs = comp_sums(v, wh, mode == 0.f);
    const float ss0 = __shfl_sync(0xffffffffu, cs.ss, b0), ss1 = __shfl_sync(0xffffffffu, cs.ss, b0 + 1),
                ss2 = __shfl_sync(0xffffffffu, cs.ss, b0 + 2);
    const float sh0 = __shfl_sync(0xffffffffu, cs.sh, b0), sh1 = __shfl_sync(0xffffffffu, cs.sh, b0 + 1),
                sh2 = __shfl_sync(0xffffffffu, cs.sh, b0 + 2);
    const float tr1 = __shfl_sync(0xffffffffu, cs.tr, b0 + 1), tr2 = __shfl_sync(0xffffffffu, cs.tr, b0 + 2);
    const float scale = scale_of(ss0, ss1, ss2, sh0, sh1, sh2, mode);
    if (lane < 3 * FDROP && i < n) {
      unsigned w[32];
      comp_features(v, fs2, sg * (1.f / scale), w);
      unsigned char* tb = reinterpret_cast<unsigned char*>(Xg) + (i / TM) * TILE_X_BYTES;
      const int rr = (int)(i % TM);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<uint4*>(tb + blk_off(rr, 8 * c + q, TM)) =
            make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
      if (c == 0) {
        unsigned wt[8];
        tail_features(f.tc, wt);
        *reinterpret_cast<uint4*>(tb + blk_off(rr, 24, TM)) = make_uint4(wt[0], wt[1], wt[2], wt[3]);
        *reinterpret_cast<uint4*>(tb + blk_off(rr, 25, TM)) = make_uint4(wt[4], wt[5], wt[6], wt[7]);
        const float trc[3] = {cs.tr, tr1, tr2};
        float* ax = auxg + i * 8;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const int d = frame_perm(f.code, cc);
          const float val = trc[cc];  // unsigned: already the grid-frame tricubic value
          if (d == 0) ax[0] = val;
          else if (d == 1) ax[1] = val;
          else ax[2] = val;
        }
        ax[3] = scale;
        ax[4] = __int_as_float(f.code);
      }
    }
  }
}

// ---- MLP forward on the 5th-generation tensor cores --------------------------------------------
// Persistent CTA per SM, 16 warps in two groups of 8.  The CTA's tiles (TM = 128 droplets each)
// alternate between the groups, so that one group's epilogues overlap the other group's MMAs.
// Per tile:
//   X tile (128 x 208 bf16, tile layout) arrives by one bulk asynchronous copy into the single X
//   buffer; the group whose layer 1 has just consumed X issues the copy of the CTA's next tile;
//   layer 1: 13 tcgen05.mma (M 128, N 128, K 16) from X and W1 into the group's TMEM columns;
//   epilogue: the group's 8 warps read the accumulators (tcgen05.ld; warp w: TMEM lanes
//   32 (w % 4), columns 64 ((w / 4) % 2)), add b1, SiLU, bf16 -> the group's H (tile layout);
//   layer 2: 8 MMAs from H and W2; epilogue as above -> H;
//   layer 3: 8 MMAs (N 16: W3 padded); 4 warps write out = tricubic + scale * os * MLP in the grid
//   frame.
// The group's leader issues its MMAs and commits them to the group's mbarrier; group barriers are
// named barriers.  Every wait is bounded (wait_limit polls, the plan's setting): a wait that runs
// out raises LD_STATUS_WAIT_TIMEOUT and the group stops; before the CTA frees its tensor memory
// and exits, one thread waits (bounded by kWaitLimitMlp) for the feature copy and the MMAs that
// are still in flight, so that nothing writes shared or tensor memory after the CTA has left.
// With `stall` set (a test of that path) each group first waits on a barrier that nothing
// completes, while the CTA's first feature copy is in flight.
constexpr int FT_THREADS = 512;
constexpr int FT_GROUP = 256;                         // threads of a group
constexpr int SM_W1 = 0;
constexpr int SM_W2 = SM_W1 + H * K1 * 2;             // 53248
constexpr int SM_W3 = SM_W2 + H * H * 2;              // + 32768
constexpr int SM_X = SM_W3 + N3P * H * 2;             // + 4096
constexpr int SM_H0 = SM_X + TILE_X_BYTES;
constexpr int SM_H1 = SM_H0 + TM * H * 2;
constexpr int SM_BIAS = SM_H1 + TM * H * 2;           // b1[128], b2[128], b3[16]
constexpr int SM_BAR = SM_BIAS + (2 * H + N3P) * 4;   // bar_x[2], bar_mma[2], bar_stall, bar_w
constexpr int SM_TMEM = SM_BAR + 6 * 8;
constexpr int SM_CNT = SM_TMEM + 16;
constexpr size_t SMEM_FWD = SM_CNT + 8 * 4;
constexpr unsigned TMEM_COLS = 512;                   // group g: columns 256 g .. 256 g + 143
constexpr unsigned kWaitLimitMlp = 1u << 24;

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(FT_GROUP) : "memory");
}

// group barrier that returns the OR of v over the group's threads (group-uniform decisions)
__device__ __forceinline__ bool group_or(int g, bool v) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((unsigned)v), "r"(1 + g), "r"(FT_GROUP)
      : "memory");
  return r != 0;
}

template <typename T>
__global__ void __launch_bounds__(FT_THREADS, 1)
k_mlp_forward_tc(const unsigned char* __restrict__ Xg, const float* __restrict__ auxg, long long n,
                 const bf16* __restrict__ packed, const float* __restrict__ params, T* __restrict__ out,
                 unsigned* __restrict__ status, unsigned wait_limit, int stall) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = warp >> 3, gw = warp & 7;             // group, warp within the group
  const bool leader = (tid & (FT_GROUP - 1)) == 0;
  float* bias = reinterpret_cast<float*>(sm + SM_BIAS);
  // copy i of the X buffer completes on bar_x[i % 2]: group g waits only on bar_x[g], so every
  // barrier's k-th wait has parity k % 2 (a fresh barrier counts parity 1 as complete)
  uint64_t* bar_x = reinterpret_cast<uint64_t*>(sm + SM_BAR);
  uint64_t* bar_mma = bar_x + 2;
  uint64_t* bar_stall = bar_x + 4;  // completed by nothing: the first wait of a stall test
  uint64_t* bar_w = bar_x + 5;      // the weights' bulk copies
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(sm + SM_TMEM);
  // drain bookkeeping: X copies issued to / waited on each bar_x, MMA commits to / waits on each
  // bar_mma; each counter has one writer (a group leader; cnt[0] leaves out the first copy, which
  // thread 0 issues before the loop) and thread 0 reads them after the final barrier
  unsigned* cnt = reinterpret_cast<unsigned*>(sm + SM_CNT);  // [x_issued 2][x_waited 2][mma_commit 2][mma_wait 2]
  // b1, b2 halved: the epilogues form h = z / 2 = fma(0.5, acc, b / 2), which is exactly
  // 0.5 * (acc + b) (halving is exact), and SiLU(z) = h + h tanh(h); b3 as is
  for (int e = tid; e < 2 * H + N3P; e += FT_THREADS)
    bias[e] = e < H ? 0.5f * params[OFF_B1 + e]
                    : (e < 2 * H ? 0.5f * params[OFF_B2 + e - H] : (e - 2 * H < N3 ? params[OFF_B3 + e - 2 * H] : 0.f));
  const long long ntiles = (n + TM - 1) / TM;
  const long long mine = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;  // CTA's tiles
  if (tid == 0) {
    mbar_init(&bar_x[0], 1);
    mbar_init(&bar_x[1], 1);
    mbar_init(&bar_mma[0], 1);
    mbar_init(&bar_mma[1], 1);
    mbar_init(bar_stall, 1);
    mbar_init(bar_w, 1);
    mbar_init_fence();
    // the weights (their tile-layout copies) and the CTA's first feature tile, as bulk copies in
    // flight together
    mbar_expect_tx(bar_w, (H * K1 + H * H + N3P * H) * 2);
    bulk_g2s(sm + SM_W1, packed + P_TW1, H * K1 * 2, bar_w);
    bulk_g2s(sm + SM_W2, packed + P_TW2, H * H * 2, bar_w);
    bulk_g2s(sm + SM_W3, packed + P_TW3, N3P * H * 2, bar_w);
    if (mine > 0) {  // the first copy is counted at the end (x_issued[0] + 1)
      mbar_expect_tx(&bar_x[0], TILE_X_BYTES);
      bulk_g2s(sm + SM_X, Xg + blockIdx.x * (long long)TILE_X_BYTES, TILE_X_BYTES, &bar_x[0]);
    }
  }
  if (tid < 8) cnt[tid] = 0u;
  if (warp == 0) {
    tmem_alloc(tmem_slot, TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();  // the barriers are initialised
  tc_fence_after();
  const unsigned tmem = *tmem_slot + 256u * (unsigned)g;
  unsigned char* Hs = sm + (g ? SM_H1 : SM_H0);
  const float os = params[OFF_OS];
  constexpr unsigned ID1 = umma_idesc_bf16(128, 128), ID3 = umma_idesc_bf16(128, N3P);
  unsigned ph = 0;
  // the weights are in shared memory before any MMA (group-uniform outcome)
  bool failed = group_or(g, !mbar_wait_bounded(bar_w, 0u, wait_limit));
  for (long long i = g; i < mine && !failed; i += 2) {
    const long long tile = blockIdx.x + i * (long long)gridDim.x;
    // the output warps' aux rows (tricubic xyz, scale, frame code) load while the layers run
    const long long orow = tile * TM + 32 * gw + lane;
    float4 ax0 = make_float4(0.f, 0.f, 0.f, 0.f);
    int code = 0;
    if (gw < 4 && orow < n) {
      ax0 = *reinterpret_cast<const float4*>(auxg + orow * 8);
      code = __float_as_int(auxg[orow * 8 + 4]);
    }
    // X of this tile (the i-th copy into the X buffer, on bar_x[g], the group's (i/2)-th wait);
    // failures are made group-uniform
    if (stall && i == g) {  // a wait on a barrier that nothing completes runs out
      failed = group_or(g, !mbar_wait_bounded(bar_stall, 0u, wait_limit));
      if (failed) break;
    }
    failed = group_or(g, !mbar_wait_bounded(&bar_x[g], (unsigned)((i >> 1) & 1), wait_limit));
    if (failed) break;
    if (leader) {
      cnt[2 + g] += 1u;
      tc_fence_after();
#pragma unroll 1
      for (int k = 0; k < K1 / 16; ++k)
        umma_bf16(tmem, umma_desc(sm + SM_X + 2 * k * (TM / 8) * 128, (TM / 8) * 128, 128),
                  umma_desc(sm + SM_W1 + 2 * k * (H / 8) * 128, (H / 8) * 128, 128), ID1, k > 0);
      umma_commit(&bar_mma[g]);
      cnt[4 + g] += 1u;
    }
    for (int layer = 0; layer < 3; ++layer) {
      failed = group_or(g, !mbar_wait_bounded(&bar_mma[g], ph, wait_limit));
      if (!failed && leader) cnt[6 + g] += 1u;
      ph ^= 1u;
      tc_fence_after();
      if (layer == 0 && leader && !failed && i + 1 < mine) {
        // layer 1 has consumed X: bring in the CTA's next tile (the other group's, on its barrier)
        cnt[g ^ 1] += 1u;
        mbar_expect_tx(&bar_x[g ^ 1], TILE_X_BYTES);
        bulk_g2s(sm + SM_X, Xg + (tile + gridDim.x) * (long long)TILE_X_BYTES, TILE_X_BYTES, &bar_x[g ^ 1]);
      }
      if (failed) break;
      if (layer < 2) {
        // epilogue: rows 32 (gw % 4) + lane, columns 64 (gw / 4) .. + 63
        const int sub = gw & 3, half = gw >> 2;
        const int row = 32 * sub + lane;
        const float* bl = bias + layer * H;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int col0 = 64 * half + 32 * cc;
          float v[32];
          tmem_ld32(tmem + ((unsigned)(32 * sub) << 16) + (unsigned)col0, v);
          const float4* b4p = reinterpret_cast<const float4*>(bl + col0);
          unsigned w[16];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            // h = fma(0.5, acc, b / 2) and SiLU = fma(h, tanh(h), h) two columns at a time (packed
            // FP32 pairs: the same roundings as the scalar forms)
            const float4 b4 = b4p[j];
            const float2 h0 = __ffma2_rn(make_float2(0.5f, 0.5f), make_float2(v[4 * j], v[4 * j + 1]),
                                         make_float2(b4.x, b4.y));
            const float2 h1 = __ffma2_rn(make_float2(0.5f, 0.5f), make_float2(v[4 * j + 2], v[4 * j + 3]),
                                         make_float2(b4.z, b4.w));
            const float2 s0 = __ffma2_rn(h0, make_float2(tanh_fast(h0.x), tanh_fast(h0.y)), h0);
            const float2 s1 = __ffma2_rn(h1, make_float2(tanh_fast(h1.x), tanh_fast(h1.y)), h1);
            w[2 * j] = pack2(s0.x, s0.y);
            w[2 * j + 1] = pack2(s1.x, s1.y);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(Hs + blk_off(row, col0 / 8 + q, TM)) =
                make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        }
        fence_proxy_async_smem();
        tc_fence_before();
        group_sync(g);
        if (leader) {
          tc_fence_after();
          if (layer == 0) {
#pragma unroll 1
            for (int k = 0; k < H / 16; ++k)
              umma_bf16(tmem, umma_desc(Hs + 2 * k * (TM / 8) * 128, (TM / 8) * 128, 128),
                        umma_desc(sm + SM_W2 + 2 * k * (H / 8) * 128, (H / 8) * 128, 128), ID1, k > 0);
          } else {
#pragma unroll 1
            for (int k = 0; k < H / 16; ++k)
              umma_bf16(tmem + 128, umma_desc(Hs + 2 * k * (TM / 8) * 128, (TM / 8) * 128, 128),
                        umma_desc(sm + SM_W3 + 2 * k * (N3P / 8) * 128, (N3P / 8) * 128, 128), ID3, k > 0);
          }
          umma_commit(&bar_mma[g]);
          cnt[4 + g] += 1u;
        }
      } else if (gw < 4) {
        float v[16];
        tmem_ld16(tmem + ((unsigned)(32 * gw) << 16) + 128u, v);
        if (orow < n) {
          const float tg[3] = {ax0.x, ax0.y, ax0.z};
#pragma unroll
          for (int c = 0; c < D_OUT; ++c) {
            const int cg = frame_perm(code, c);
            const float y = v[c] + bias[2 * H + c];
            const float t = cg == 0 ? tg[0] : (cg == 1 ? tg[1] : tg[2]);
            out[3 * orow + cg] = T(t + ax0.w * (os * frame_sign(code, cg) * y));
          }
        }
      }
    }
    tc_fence_before();
    group_sync(g);  // the group's TMEM and H are free for its next tile
  }
  if (failed && (tid & (FT_GROUP - 1)) == 0) atomicOr(status, LD_STATUS_WAIT_TIMEOUT);
  tc_fence_before();
  const bool any_failed = __syncthreads_or(failed) != 0;
  tc_fence_after();
  if (any_failed) {
    // a group stopped early: copies and MMAs it (or the other group) issued may still be in
    // flight; wait for each barrier's outstanding completion (the k-th completion of a barrier
    // has parity k % 2) before the tensor memory is freed and the shared memory released
    if (tid == 0) {
      mbar_wait_bounded(bar_w, 0u, kWaitLimitMlp);  // the weights' copies
      for (int b = 0; b < 2; ++b) {
        const unsigned x_issued = cnt[b] + (b == 0 && mine > 0 ? 1u : 0u);
        if (x_issued > cnt[2 + b]) mbar_wait_bounded(&bar_x[b], cnt[2 + b] & 1u, kWaitLimitMlp);
        if (cnt[4 + b] > cnt[6 + b]) mbar_wait_bounded(&bar_mma[b], cnt[6 + b] & 1u, kWaitLimitMlp);
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (warp == 0) tmem_dealloc(*tmem_slot, TMEM_COLS);
}

// ---- training samples ------------------------------------------------------------------------------
// For sample s: point = grid point idx[s] + shift (in grid units), exact velocity = ue (planar
// (3, N^3)) at idx[s] (ue is the field phase-shifted by `shift`), features from the unshifted
// interleaved field u4.  Writes X row, target T = (exact - tricubic)/(scale os) in the point's
// canonical frame, tricubic (grid frame) and scale.
template <typename T>
__global__ void k_mlp_samples(const vec4<T>* __restrict__ u4, const T* __restrict__ ue, int N, double L,
                              const long long* __restrict__ idx, long long ns, double sx, double sy, double sz,
                              const float* __restrict__ params, bf16* __restrict__ X, float* __restrict__ Tg,
                              float* __restrict__ aux) {
  const long long N3g = (long long)N * N * N;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < ns; s += (long long)gridDim.x * blockDim.x) {
    const long long j = idx[s];
    const long long jx = j / ((long long)N * N), jy = (j / N) % N, jz = j % N;
    const double dx = L / N;
    const double px = (jx + sx) * dx, py = (jy + sy) * dx, pz = (jz + sz) * dx;
    float st[192], tric[3], tric_can[3];
    int code;
    const float scale = point_features<T>(u4, N, L, px, py, pz, params, st, X + s * K1, tric, code, tric_can);
    const float os = params[OFF_OS];
    for (int cc = 0; cc < 3; ++cc) {  // target in the canonical frame
      const int cg = frame_perm(code, cc);
      const float ex = frame_sign(code, cg) * float(ue[cg * N3g + j]);
      Tg[s * 3 + cc] = (ex - tric_can[cc]) / (scale * os);
    }
    for (int c = 0; c < 3; ++c) aux[s * 4 + c] = tric[c];
    aux[s * 4 + 3] = scale;
  }
}

// uk * exp(i k . shift dx): the spectrum of the field translated by -shift (its values at grid
// point j are the field's values at x_j + shift).
template <typename T>
__global__ void k_phase_shift(const ld::cplx<T>* __restrict__ in, ld::cplx<T>* __restrict__ out, long long cs, int kc,
                              int My, int Mzp, double ax, double ay, double az) {
  const long long total = 3 * cs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e % cs;
    const int ix = (int)(r / ((long long)My * Mzp));
    const int iy = (int)((r / Mzp) % My);
    const int kz = (int)(r % Mzp);
    const int kx = ix <= kc ? ix : ix - My, ky = iy <= kc ? iy : iy - My;
    double sn, cn;
    sincos(ax * kx + ay * ky + az * kz, &sn, &cn);
    const ld::cplx<T> v = in[e];
    out[e] = ld::cmk(T(v.x * cn - v.y * sn), T(v.x * sn + v.y * cn));
  }
}

// ---- training on the 5th-generation tensor cores -----------------------------------------------
// One CTA of 512 threads takes TBT = 128 samples of a batch (the M of every MMA) through the
// forward and backward passes and writes its gradient partial; the partials are summed in a fixed
// order afterwards (deterministic):
//   forward  Z1 = X W1 + b1, H1 = bf16(SiLU(Z1)), Z2 = H1 W2 + b2, H2 = bf16(SiLU(Z2)),
//            Y = H2 W3 + b3 (the MMAs and epilogue arithmetic of the inference kernel);
//   dY       = 2 w (Y - T) / B on valid rows (zero on the padding rows of a partial tile);
//   dZ2      = (dY W3^T) * SiLU'(Z2),  dZ1 = dH1 * SiLU'(Z1)   (FP32, in the epilogues);
//   dW3 = H2^T dY, dW2 = H1^T dZ2, dH1 = dZ2 W2^T, dW1 = X^T dZ1 on the tensor cores.
// The weight gradients contract over the samples: their operands are the shared tiles that the
// forward MMAs read K-major (samples as rows), read MN-major (samples along K).  dY, dZ2 and dZ1
// enter as two BF16 parts, hi = bf16(d) and lo = bf16(d - hi), accumulated into the same FP32
// sums, so that the products carry about 16 bits of the FP32 values; X, H1, H2 and the weights are
// BF16 already.  Bias gradients are column sums of the FP32 values: a butterfly over the 32 rows
// of a warp, then the four row quadrants in order.
// Warp w of the epilogues: TMEM lanes (samples, or weight rows for the gradients) 32 (w % 4) ..
// + 31, columns 32 (w / 4) .. + 31.
// TMEM columns (512): Z1 0..127, later dW1 rows 0..127; Z2 128..255, later dH1, later dW1 rows
// 80..207; Y 256..271, later dW3; dW2 384..511.
// Shared memory: W1 until layer 1 completes, then H1 | H2; W2; X; W3 until layer 3 completes,
// then dZ hi | lo (dZ2, later dZ1); dY hi | lo (16 x 128 each).  The weights arrive as three bulk
// copies of their tile-layout copies, the samples' rows as 16-byte asynchronous copies; dW2 and
// dW1 leave as one bulk store per row from shared memory, the small gradients as plain stores.
// Every wait is bounded (kWaitLimitMlp polls); a wait that runs out makes the CTA wait (bounded)
// for the MMAs in flight, write NaN as its loss partial (the batch loss, and so the epoch loss,
// become NaN) and free its tensor memory.
constexpr int TR_THREADS = 512;
constexpr int TR_PARTS = TR_THREADS / 128;            // column parts of the epilogues (4)
constexpr int TR_COLS = H / TR_PARTS;                 // columns of a warp in the epilogues (32)
constexpr int TBT = 128;                              // samples per CTA
constexpr int TS_H1 = 0;                              // W1 (53248 B) until layer 1 completes
constexpr int TS_H2 = TS_H1 + TBT * H * 2;            // 32768
constexpr int TS_W2 = TS_H2 + TBT * H * 2;            // 65536
constexpr int TS_X = TS_W2 + H * H * 2;               // 98304
constexpr int TS_D = TS_X + TBT * K1 * 2;             // 151552: W3 until layer 3 completes, then dZ hi
constexpr int TS_DLO = TS_D + TBT * H * 2;            // 184320
constexpr int TS_Y = TS_DLO + TBT * H * 2;            // 217088: dY hi
constexpr int TS_YLO = TS_Y + N3P * TBT * 2;          // 221184
constexpr int TS_BIAS = TS_YLO + N3P * TBT * 2;       // 225280: b1 / 2, b2 / 2, b3 (272 floats)
constexpr int TS_DYF = TS_BIAS + (2 * H + N3P) * 4;   // 226368: dY FP32 [128][4]
constexpr int TS_CS = TS_DYF + TBT * 4 * 4;           // 228416: column sums of the quadrants [4][128]
constexpr int TS_CS3 = TS_CS + 4 * H * 4;             // 230464: dY column sums [4][4]
constexpr int TS_LOSS = TS_CS3 + 16 * 4;              // 230528: loss of warps 0..3
constexpr int TS_BAR = TS_LOSS + 8 * 4;               // 230560
constexpr int TS_TMEM = TS_BAR + 8;                   // 230568
constexpr int TS_W3F = TS_TMEM + 8;                   // 230576: W3 columns 0..2 as FP32 [3][128]
constexpr int TS_WBAR = TS_W3F + D_OUT * H * 4;       // 232112: the weights' bulk copies
constexpr size_t SMEM_TRAIN_TC = TS_WBAR + 8;         // 232120
// FP32 gradient rows staged for bulk stores, 16 bytes of padding per row (the rows of a warp's
// 16-byte writes fall on distinct bank groups): dW2 over H1 | H2 | W2, dW1 over X | dZ
constexpr int ST_ROW = H * 4 + 16;
static_assert(H * ST_ROW <= TS_X && K1 * ST_ROW <= TS_Y - TS_X, "gradient staging");
static_assert(SMEM_TRAIN_TC <= 227 * 1024, "training kernel exceeds shared memory");
static_assert(H * K1 * 2 <= TS_W2 && N3P * H * 2 <= TBT * H * 2, "W1 / W3 overlays");
constexpr unsigned T_Z1 = 0, T_Z2 = 128, T_Y = 256, T_DW2 = 384;

// h = fma(0.5, acc, b / 2) (= z / 2 exactly) and SiLU(z) = fma(h, tanh(h), h) on 32 columns, as the
// inference epilogue computes them, packed to 16 BF16 pairs
__device__ __forceinline__ void silu_pack32(const float (&v)[32], const float* bh, unsigned (&w)[16]) {
  const float4* b4p = reinterpret_cast<const float4*>(bh);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float4 b4 = b4p[j];
    const float2 h0 = __ffma2_rn(make_float2(0.5f, 0.5f), make_float2(v[4 * j], v[4 * j + 1]), make_float2(b4.x, b4.y));
    const float2 h1 =
        __ffma2_rn(make_float2(0.5f, 0.5f), make_float2(v[4 * j + 2], v[4 * j + 3]), make_float2(b4.z, b4.w));
    const float2 s0 = __ffma2_rn(h0, make_float2(tanh_fast(h0.x), tanh_fast(h0.y)), h0);
    const float2 s1 = __ffma2_rn(h1, make_float2(tanh_fast(h1.x), tanh_fast(h1.y)), h1);
    w[2 * j] = pack2(s0.x, s0.y);
    w[2 * j + 1] = pack2(s1.x, s1.y);
  }
}

// 32 FP32 values of one row -> the row's hi | lo BF16 parts in the tile layout (4 16-byte chunks each)
__device__ __forceinline__ void store_split32(const float (&d)[32], unsigned char* hi, unsigned char* lo, int row,
                                              int kc0) {
  unsigned wh[16], wl[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(d[2 * j], d[2 * j + 1]);
    const float2 hf = __bfloat1622float2(h);
    wh[j] = *reinterpret_cast<const unsigned*>(&h);
    wl[j] = pack2(d[2 * j] - hf.x, d[2 * j + 1] - hf.y);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    *reinterpret_cast<uint4*>(hi + blk_off(row, kc0 + c, TBT)) = make_uint4(wh[4 * c], wh[4 * c + 1], wh[4 * c + 2], wh[4 * c + 3]);
    *reinterpret_cast<uint4*>(lo + blk_off(row, kc0 + c, TBT)) = make_uint4(wl[4 * c], wl[4 * c + 1], wl[4 * c + 2], wl[4 * c + 3]);
  }
}

// Column sums over the 32 rows (lanes) of a warp: lane l returns the sum of v[l] over the lanes
// (recursive halving: each step keeps half of the columns and adds the partner lane's half;
// 31 shuffles, a fixed order).
__device__ __forceinline__ float warp_colsum32(const float (&v)[32], int lane) {
  float a[16], b[8], c[4], d[2];
  const bool u16 = lane & 16, u8 = lane & 8, u4 = lane & 4, u2 = lane & 2, u1 = lane & 1;
#pragma unroll
  for (int j = 0; j < 16; ++j)
    a[j] = (u16 ? v[16 + j] : v[j]) + __shfl_xor_sync(0xffffffffu, u16 ? v[j] : v[16 + j], 16);
#pragma unroll
  for (int j = 0; j < 8; ++j) b[j] = (u8 ? a[8 + j] : a[j]) + __shfl_xor_sync(0xffffffffu, u8 ? a[j] : a[8 + j], 8);
#pragma unroll
  for (int j = 0; j < 4; ++j) c[j] = (u4 ? b[4 + j] : b[j]) + __shfl_xor_sync(0xffffffffu, u4 ? b[j] : b[4 + j], 4);
#pragma unroll
  for (int j = 0; j < 2; ++j) d[j] = (u2 ? c[2 + j] : c[j]) + __shfl_xor_sync(0xffffffffu, u2 ? c[j] : c[2 + j], 2);
  return (u1 ? d[1] : d[0]) + __shfl_xor_sync(0xffffffffu, u1 ? d[0] : d[1], 1);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Programmatic dependent launch: the next kernel in the stream may start (its CTAs wait in
// grid_dep_wait until this grid has completed and its writes are visible); both are no-ops for a
// kernel launched without the attribute.
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// 16-byte asynchronous copy global -> shared; bytes < 16 zero-fills the rest (0: no read)
__device__ __forceinline__ void cp_async16(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes)
               : "memory");
}

// every thread waits for the MMAs committed to bar (bounded); the outcome is made block-uniform
__device__ __forceinline__ bool train_wait(uint64_t* bar, unsigned& ph) {
  const bool ok = mbar_wait_bounded(bar, ph, kWaitLimitMlp);
  ph ^= 1u;
  const bool all_ok = __syncthreads_or(!ok) == 0;
  tc_fence_after();
  return all_ok;
}

__device__ __forceinline__ void train_sync() {
  fence_proxy_async_smem();  // the epilogue's shared writes are read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// Xg (n, K1) bf16 rows, Tg (n, 3), Wg (n) or null; sample r of the batch is row order[r] (or r
// when order is null); nb samples.
__global__ void __launch_bounds__(TR_THREADS, 1)
k_mlp_train_tc(const bf16* __restrict__ Xg, const float* __restrict__ Tg, const float* __restrict__ Wg,
               const unsigned* __restrict__ order, long long nb, float inv_norm, const bf16* __restrict__ packed,
               const float* __restrict__ params, float* __restrict__ gpart, float* __restrict__ lpart) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3, part = warp >> 2;
  const int row = 32 * q + lane;  // the thread's TMEM lane in the epilogues
  const long long r0 = (long long)blockIdx.x * TBT;
  float* bias = reinterpret_cast<float*>(sm + TS_BIAS);
  float* dyf = reinterpret_cast<float*>(sm + TS_DYF);
  float* cs = reinterpret_cast<float*>(sm + TS_CS);
  float* cs3 = reinterpret_cast<float*>(sm + TS_CS3);
  float* lw = reinterpret_cast<float*>(sm + TS_LOSS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + TS_BAR);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(sm + TS_TMEM);
  float* w3s = reinterpret_cast<float*>(sm + TS_W3F);
  uint64_t* wbar = reinterpret_cast<uint64_t*>(sm + TS_WBAR);
  float* G = gpart + (long long)blockIdx.x * N_PARAMS;
  grid_dep_launch();
  // the CTA's samples gathered by order (16-byte asynchronous copies, all in flight together;
  // rows past nb: zero fill); thread t copies chunks of sample t % 128.  X, T, W and order are
  // not written by the kernels of a training step: they load before the wait for the previous
  // step's parameter update (programmatic dependent launch)
  {
    const int r = tid % TBT;
    const bool valid = r0 + r < nb;
    const long long src = valid ? (order ? (long long)order[r0 + r] : r0 + r) : 0;
    const bf16* xrow = Xg + src * K1;
#pragma unroll
    for (int kc = tid / TBT; kc < K1 / 8; kc += TR_THREADS / TBT)
      cp_async16(sm + TS_X + blk_off(r, kc, TBT), xrow + 8 * kc, valid ? 16u : 0u);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  grid_dep_wait();  // the parameters and their packed copies are final; gpart may be written
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(wbar, 1);
    mbar_init_fence();
    mbar_expect_tx(wbar, (H * K1 + H * H + N3P * H) * 2);
    bulk_g2s(sm + TS_H1, packed + P_TW1, H * K1 * 2, wbar);
    bulk_g2s(sm + TS_W2, packed + P_TW2, H * H * 2, wbar);
    bulk_g2s(sm + TS_D, packed + P_TW3, N3P * H * 2, wbar);
  }
  for (int e = tid; e < 2 * N3P * TBT * 2 / 16; e += TR_THREADS)  // dY hi | lo: columns 3..15 stay zero
    reinterpret_cast<uint4*>(sm + TS_Y)[e] = make_uint4(0u, 0u, 0u, 0u);
  for (int e = tid; e < 2 * H + N3P; e += TR_THREADS)
    bias[e] = e < H ? 0.5f * params[OFF_B1 + e]
                    : (e < 2 * H ? 0.5f * params[OFF_B2 + e - H] : (e - 2 * H < N3 ? params[OFF_B3 + e - 2 * H] : 0.f));
  for (int e = tid; e < D_OUT * H; e += TR_THREADS)  // the BF16 W3 of the forward, column-major
    w3s[e] = __bfloat162float(packed[P_W3N + (e % H) * N3 + e / H]);
  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  __syncthreads();  // the barriers are initialised
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  const bool wok = mbar_wait_bounded(wbar, 0u, kWaitLimitMlp);
  fence_proxy_async_smem();
  tc_fence_before();
  bool ok = __syncthreads_or(!wok) == 0;
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned tl = tmem + ((unsigned)(32 * q) << 16);  // the warp's TMEM lanes
  constexpr unsigned CM = (TBT / 8) * 128;                // chunk stride of a 128-row tile (2048 B)
  constexpr unsigned IDK = umma_idesc_bf16(128, 128);     // A and B K-major
  constexpr unsigned ID3 = umma_idesc_bf16(128, N3P);
  constexpr unsigned IDW3 = ID3 | (1u << 15);             // A MN-major
  constexpr unsigned IDH = IDK | (1u << 16);              // B MN-major
  constexpr unsigned IDW = IDK | (1u << 15) | (1u << 16); // A and B MN-major
  unsigned ph = 0;
  do {
    if (!ok) break;
    // layer 1: Z1 = X W1
    if (tid == 0) {
#pragma unroll 1
      for (int k = 0; k < K1 / 16; ++k)
        umma_bf16(tmem + T_Z1, umma_desc(sm + TS_X + 2 * k * CM, CM, 128),
                  umma_desc(sm + TS_H1 + 2 * k * (H / 8) * 128, (H / 8) * 128, 128), IDK, k > 0);
      umma_commit(bar);
    }
    if (!(ok = train_wait(bar, ph))) break;
    // H1 over W1 (consumed)
#pragma unroll
    for (int cc = 0; cc < TR_COLS / 32; ++cc) {
      const int col0 = TR_COLS * part + 32 * cc;
      float v[32];
      unsigned w[16];
      tmem_ld32(tl + T_Z1 + col0, v);
      silu_pack32(v, bias + col0, w);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4*>(sm + TS_H1 + blk_off(row, col0 / 8 + c, TBT)) =
            make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
    }
    train_sync();
    // layer 2: Z2 = H1 W2
    if (tid == 0) {
#pragma unroll 1
      for (int k = 0; k < H / 16; ++k)
        umma_bf16(tmem + T_Z2, umma_desc(sm + TS_H1 + 2 * k * CM, CM, 128),
                  umma_desc(sm + TS_W2 + 2 * k * (H / 8) * 128, (H / 8) * 128, 128), IDK, k > 0);
      umma_commit(bar);
    }
    if (!(ok = train_wait(bar, ph))) break;
#pragma unroll
    for (int cc = 0; cc < TR_COLS / 32; ++cc) {
      const int col0 = TR_COLS * part + 32 * cc;
      float v[32];
      unsigned w[16];
      tmem_ld32(tl + T_Z2 + col0, v);
      silu_pack32(v, bias + H + col0, w);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4*>(sm + TS_H2 + blk_off(row, col0 / 8 + c, TBT)) =
            make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
    }
    train_sync();
    // layer 3: Y = H2 W3
    if (tid == 0) {
#pragma unroll 1
      for (int k = 0; k < H / 16; ++k)
        umma_bf16(tmem + T_Y, umma_desc(sm + TS_H2 + 2 * k * CM, CM, 128),
                  umma_desc(sm + TS_D + 2 * k * (N3P / 8) * 128, (N3P / 8) * 128, 128), ID3, k > 0);
      umma_commit(bar);
    }
    if (!(ok = train_wait(bar, ph))) break;
    // dY, the loss and db3 (warps 0..3: one sample per thread)
    if (part == 0) {
      float v[16];
      tmem_ld16(tl + T_Y, v);
      const long long gr = r0 + row;
      const bool valid = gr < nb;
      const long long src = valid ? (order ? (long long)order[gr] : gr) : 0;
      const float wr = (valid && Wg) ? Wg[src] : 1.f;
      float d[3], ls = 0.f;
#pragma unroll
      for (int c = 0; c < D_OUT; ++c) {
        d[c] = 0.f;
        if (valid) {
          const float e = (v[c] + bias[2 * H + c]) - Tg[src * 3 + c];
          ls += wr * e * e;
          d[c] = 2.f * e * wr * inv_norm;
        }
        dyf[row * 4 + c] = d[c];
        // dY as the B operand of dW3 (N = output column, K = sample): 16-row K-major tile
        const bf16 hi = __float2bfloat16_rn(d[c]);
        const bf16 lo = __float2bfloat16_rn(d[c] - __bfloat162float(hi));
        const int off = blk_off(c, row >> 3, N3P) + (row & 7) * 2;
        *reinterpret_cast<bf16*>(sm + TS_Y + off) = hi;
        *reinterpret_cast<bf16*>(sm + TS_YLO + off) = lo;
      }
      ls = warp_sum(ls);
      const float s0 = warp_sum(d[0]), s1 = warp_sum(d[1]), s2 = warp_sum(d[2]);
      if (lane == 0) {
        lw[q] = ls;
        cs3[4 * q] = s0;
        cs3[4 * q + 1] = s1;
        cs3[4 * q + 2] = s2;
      }
    }
    __syncthreads();
    // dZ2 = (dY W3^T) * SiLU'(Z2): hi | lo over the W3 tile (consumed); db2 quadrant sums
    {
      const float dy0 = dyf[row * 4], dy1 = dyf[row * 4 + 1], dy2 = dyf[row * 4 + 2];
#pragma unroll
      for (int cc = 0; cc < TR_COLS / 32; ++cc) {
        const int col0 = TR_COLS * part + 32 * cc;
        float v[32];
        tmem_ld32(tl + T_Z2 + col0, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int i = col0 + j;
          float s = dy0 * w3s[i];
          s = fmaf(dy1, w3s[H + i], s);
          s = fmaf(dy2, w3s[2 * H + i], s);
          const float z = 2.f * fmaf(0.5f, v[j], bias[H + i]);  // the forward's pre-activation, exactly
          v[j] = s * dsilu(z);
        }
        store_split32(v, sm + TS_D, sm + TS_DLO, row, col0 / 8);
        cs[q * H + col0 + lane] = warp_colsum32(v, lane);
      }
    }
    train_sync();
    // dW3 = H2^T dY, dH1 = dZ2 W2^T, dW2 = H1^T dZ2, each from the hi and the lo part
    if (tid == 0) {
#pragma unroll 1
      for (int k = 0; k < TBT / 16; ++k)
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          const unsigned char* dz = sm + (part ? TS_DLO : TS_D);
          const unsigned char* dy = sm + (part ? TS_YLO : TS_Y);
          const unsigned acc = (k > 0 || part > 0) ? 1u : 0u;
          // A: H2 with the samples along K (MN-major); B: the dY tile (K-major)
          umma_bf16(tmem + T_Y, umma_desc(sm + TS_H2 + 2 * k * 128, 128, CM),
                    umma_desc(dy + 2 * k * (N3P / 8) * 128, (N3P / 8) * 128, 128), IDW3, acc);
          // A: dZ2 (K = hidden column o, K-major); B: the W2 tile (rows o) read with N = i (MN-major)
          umma_bf16(tmem + T_Z2, umma_desc(dz + 2 * k * CM, CM, 128), umma_desc(sm + TS_W2 + 2 * k * 128, 128, CM),
                    IDH, acc);
          // A: H1, B: dZ2, both with the samples along K (MN-major)
          umma_bf16(tmem + T_DW2, umma_desc(sm + TS_H1 + 2 * k * 128, 128, CM), umma_desc(dz + 2 * k * 128, 128, CM),
                    IDW, acc);
        }
      umma_commit(bar);
    }
    static_assert(TR_THREADS >= 256 + (N_PARAMS - OFF_FS), "thread ranges of the partial writes");
    if (tid >= 128 && tid < 256) {
      const int o = tid - 128;
      G[OFF_B2 + o] = ((cs[o] + cs[H + o]) + cs[2 * H + o]) + cs[3 * H + o];
    } else if (tid >= 32 && tid < 32 + N3) {
      const int c = tid - 32;
      G[OFF_B3 + c] = c < D_OUT ? ((cs3[c] + cs3[4 + c]) + cs3[8 + c]) + cs3[12 + c] : 0.f;
    } else if (tid >= 256 && tid < 256 + (N_PARAMS - OFF_FS)) {
      G[OFF_FS + tid - 256] = 0.f;  // the scales are not trained
    } else if (tid == 64) {
      lpart[blockIdx.x] = ((lw[0] + lw[1]) + lw[2]) + lw[3];
    }
    if (!(ok = train_wait(bar, ph))) break;
    // dZ1 = dH1 * SiLU'(Z1): hi | lo over dZ2 (consumed); db1 quadrant sums; dW2 and dW3 out
#pragma unroll 1
    for (int cc = 0; cc < TR_COLS / 32; ++cc) {
      const int col0 = TR_COLS * part + 32 * cc;
      float v[32], a1[32];
      tmem_ld32(tl + T_Z2 + col0, v);
      tmem_ld32(tl + T_Z1 + col0, a1);
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] *= dsilu(2.f * fmaf(0.5f, a1[j], bias[col0 + j]));
      store_split32(v, sm + TS_D, sm + TS_DLO, row, col0 / 8);
      cs[q * H + col0 + lane] = warp_colsum32(v, lane);
      tmem_ld32(tl + T_DW2 + col0, a1);  // dW2 row i = row, columns o: staged over H1 | H2 | W2 (consumed)
      float4* s4 = reinterpret_cast<float4*>(sm + row * ST_ROW + col0 * 4);
#pragma unroll
      for (int j = 0; j < 8; ++j) s4[j] = make_float4(a1[4 * j], a1[4 * j + 1], a1[4 * j + 2], a1[4 * j + 3]);
    }
    if (part == 0) {
      float v[16];
      tmem_ld16(tl + T_Y, v);  // dW3 row i = row, columns c (3..7 are zero)
      float4* g4 = reinterpret_cast<float4*>(G + OFF_W3 + row * N3);
      g4[0] = make_float4(v[0], v[1], v[2], v[3]);
      g4[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    train_sync();
    if (tid < H) {  // dW2 rows out
      bulk_s2g(G + OFF_W2 + tid * H, sm + tid * ST_ROW, H * 4);
      bulk_commit();
    }
    // dW1 = X^T dZ1: rows k 0..127 (X chunks 0..15) and 80..207 (chunks 10..25)
    if (tid == 0) {
#pragma unroll 1
      for (int k = 0; k < TBT / 16; ++k)
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          const unsigned char* dz = sm + (part ? TS_DLO : TS_D);
          const unsigned acc = (k > 0 || part > 0) ? 1u : 0u;
          umma_bf16(tmem + T_Z1, umma_desc(sm + TS_X + 2 * k * 128, 128, CM), umma_desc(dz + 2 * k * 128, 128, CM),
                    IDW, acc);
          umma_bf16(tmem + T_Z2, umma_desc(sm + TS_X + 10 * CM + 2 * k * 128, 128, CM),
                    umma_desc(dz + 2 * k * 128, 128, CM), IDW, acc);
        }
      umma_commit(bar);
    }
    if (tid >= 128 && tid < 256) {
      const int o = tid - 128;
      G[OFF_B1 + o] = ((cs[o] + cs[H + o]) + cs[2 * H + o]) + cs[3 * H + o];
    }
    if (!(ok = train_wait(bar, ph))) break;
    {
      // parts 0 .. TR_PARTS/2 - 1: rows 0..127; the others: rows 80..207, stored from 128
      constexpr int HP = TR_PARTS / 2, CW = H / HP;
      const bool upper = part >= HP;
      const int kr = upper ? 80 + row : row;  // the thread's dW1 row
      const unsigned tc = (upper ? T_Z2 : T_Z1) + CW * (part % HP);
      const bool st = !upper || kr >= 128;
#pragma unroll 1
      for (int cc = 0; cc < CW / 32; ++cc) {
        float v[32];
        tmem_ld32(tl + tc + 32 * cc, v);
        if (st) {  // staged over X | dZ (consumed)
          float4* s4 = reinterpret_cast<float4*>(sm + TS_X + kr * ST_ROW + (CW * (part % HP) + 32 * cc) * 4);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            s4[j] = kr < D_IN ? make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3])
                              : make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid < K1) {  // dW1 rows out
      bulk_s2g(G + OFF_W1 + tid * H, sm + TS_X + tid * ST_ROW, H * 4);
      bulk_commit();
    }
  } while (false);
  if (!ok && tid == 0) {
    mbar_wait_bounded(bar, ph ^ 1u, kWaitLimitMlp);  // the commit that was not seen
    mbar_wait_bounded(wbar, 0u, kWaitLimitMlp);      // the weights' copies
  }
  bulk_wait_all();  // this thread's bulk stores have left shared memory
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!ok && tid == 0) lpart[blockIdx.x] = __int_as_float(0x7fc00000);
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// sum_b gpart[b][e] in the order b = 0, 1, ..., with 32 loads in flight at a time
__device__ __forceinline__ float sum_partials(const float* __restrict__ gpart, int nblk, int e) {
  float s = 0.f;
  for (int b0 = 0; b0 < nblk; b0 += 32) {
    float t[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) t[j] = b0 + j < nblk ? gpart[(long long)(b0 + j) * N_PARAMS + e] : 0.f;
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (b0 + j < nblk) s += t[j];
  }
  return s;
}


// Fixed-order sum of the per-CTA partials: grad[e] = sum_b gpart[b][e]; loss = sum_b lpart[b] / norm.
__global__ void k_mlp_reduce(const float* __restrict__ gpart, const float* __restrict__ lpart, int nblk,
                             float* __restrict__ grad, float* __restrict__ loss, float inv_norm) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N_PARAMS; e += gridDim.x * blockDim.x)
    grad[e] = sum_partials(gpart, nblk, e);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float l = 0.f;
    for (int b = 0; b < nblk; ++b) l += lpart[b];
    *loss = l * inv_norm;
  }
}

// Adam on the FP32 master weight e (gradient gg); padded rows/columns stay zero.  Returns false
// for a padded entry.
__device__ __forceinline__ bool adam_one(int e, float gg, float* __restrict__ p, float* __restrict__ m,
                                         float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                                         float c2) {
  bool pad = false;
  if (e < OFF_B1) pad = (e - OFF_W1) / H >= D_IN;
  else if (e >= OFF_W3 && e < OFF_B3) pad = (e - OFF_W3) % N3 >= D_OUT;
  else if (e >= OFF_B3) pad = (e - OFF_B3) >= D_OUT;
  if (pad) {
    p[e] = 0.f;
    return false;
  }
  const float mm = b1 * m[e] + (1.f - b1) * gg;
  const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
  m[e] = mm;
  v[e] = vv;
  p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  return true;
}

__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < OFF_FS; e += gridDim.x * blockDim.x)  // scales: fixed
    adam_one(e, g[e], p, m, v, lr, b1, b2, eps, c1, c2);
}

// One training step after k_mlp_train_tc: the fixed-order sum of the CTA partials (as
// k_mlp_reduce), Adam, and the BF16 copies of each changed weight written where k_mlp_pack puts
// them (its zero padding stays); thread 0 of block 0 adds the batch loss to *loss_acc.
__global__ void k_mlp_reduce_adam(const float* __restrict__ gpart, const float* __restrict__ lpart, int nblk,
                                  float inv_norm, float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                  bf16* __restrict__ q, float lr, float b1, float b2, float eps, float c1, float c2,
                                  float* __restrict__ loss_acc) {
  grid_dep_launch();
  grid_dep_wait();  // the training kernel's partials are complete
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < OFF_FS; e += gridDim.x * blockDim.x) {
    const float gg = sum_partials(gpart, nblk, e);
    if (!adam_one(e, gg, p, m, v, lr, b1, b2, eps, c1, c2)) continue;
    const bf16 w = __float2bfloat16_rn(p[e]);
    if (e < OFF_B1) {
      const int k = (e - OFF_W1) / H, o = (e - OFF_W1) % H;
      q[P_W1T + o * KP1 + k] = w;
      q[P_TW1 + tile_elem(o, k, H)] = w;
    } else if (e >= OFF_W2 && e < OFF_B2) {
      const int i = (e - OFF_W2) / H, o = (e - OFF_W2) % H;
      q[P_W2T + o * KP2 + i] = w;
      q[P_W2N + i * KP2 + o] = w;
      q[P_TW2 + tile_elem(o, i, H)] = w;
    } else if (e >= OFF_W3 && e < OFF_B3) {
      const int i = (e - OFF_W3) / N3, c = (e - OFF_W3) % N3;
      q[P_W3T + c * KP2 + i] = w;
      q[P_W3N + i * N3 + c] = w;
      q[P_TW3 + tile_elem(c, i, N3P)] = w;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float l = 0.f;
    for (int b = 0; b < nblk; ++b) l += lpart[b];
    *loss_acc = __fadd_rn(*loss_acc, __fmul_rn(l, inv_norm));  // as the batch loss of k_mlp_reduce, then added
  }
}

// Droplet stage with the fluid velocity at the stage position given (the learned interpolation
// evaluates it in a separate launch): the arithmetic of k_droplet_stage without the gather.
template <typename T>
__global__ void k_droplet_given(int stage, const T* __restrict__ up, double* __restrict__ pos, T* __restrict__ vel,
                                const T* __restrict__ tau, T* __restrict__ a1, long long n, double h, T g) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
    const T it = T(1) / tau[i];
    if (stage == 1) {
      a1[3 * i] = (up[3 * i] - vx) * it;
      a1[3 * i + 1] = (up[3 * i + 1] - vy) * it;
      a1[3 * i + 2] = (up[3 * i + 2] - vz) * it - g;
    } else {
      const T ax = a1[3 * i], ay = a1[3 * i + 1], az = a1[3 * i + 2];
      const T hh = T(h);
      const T sx = vx + hh * ax, sy = vy + hh * ay, sz = vz + hh * az;
      const T bx = (up[3 * i] - sx) * it, by = (up[3 * i + 1] - sy) * it, bz = (up[3 * i + 2] - sz) * it - g;
      pos[3 * i] += 0.5 * h * (double(vx) + double(sx));
      pos[3 * i + 1] += 0.5 * h * (double(vy) + double(sy));
      pos[3 * i + 2] += 0.5 * h * (double(vz) + double(sz));
      vel[3 * i] = vx + T(0.5) * hh * (ax + bx);
      vel[3 * i + 1] = vy + T(0.5) * hh * (ay + by);
      vel[3 * i + 2] = vz + T(0.5) * hh * (az + bz);
    }
  }
}

// xs = x + h v (the stage-2 position of the Heun step)
template <typename T>
__global__ void k_droplet_predict(const double* __restrict__ pos, const T* __restrict__ vel, long long n, double h,
                                  double* __restrict__ xs) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 3 * n; e += (long long)gridDim.x * blockDim.x)
    xs[e] = pos[e] + h * double(vel[e]);
}

// planar (3, M) -> interleaved (M, 4) with a zero fourth component
template <typename T>
__global__ void k_interleave3(const T* __restrict__ in, vec4<T>* __restrict__ out, long long m) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    out[i] = mk4<T>(in[i], in[m + i], in[2 * m + i], T(0));
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

inline int gridn(long long n, int th) {
  long long b = (n + th - 1) / th;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" {

int ld_mlp_sizes(int64_t* n_params, int64_t* n_packed, int32_t* k_in, int32_t* batch_tile) {
  if (n_params) *n_params = N_PARAMS;
  if (n_packed) *n_packed = N_PACKED;
  if (k_in) *k_in = K1;
  if (batch_tile) *batch_tile = TBT;
  return LD_OK;
}

int ld_mlp_pack(const float* params, void* packed, void* stream) {
  if (!params || !packed) return ld_fail(LD_ERR_ARG, "ld_mlp_pack: bad arguments");
  k_mlp_pack<<<gridn(N_PACKED, 256), 256, 0, (cudaStream_t)stream>>>(params, (bf16*)packed);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_mlp_infer(ld_plan* p, const void* u4, const double* pos, int64_t n, const void* packed, const float* params,
                 void* out, void* stream) {
  return ld_mlp_infer_ws(p, u4, pos, n, packed, params, out, nullptr, 0, stream);
}

int64_t ld_mlp_infer_workspace_bytes(int64_t n) {
  const long long tiles = (n + TM - 1) / TM;
  return tiles * (long long)TILE_X_BYTES + tiles * TM * (long long)sizeof(float) * 8;
}

int ld_mlp_infer_ws(ld_plan* p, const void* u4, const double* pos, int64_t n, const void* packed, const float* params,
                    void* out, void* work, int64_t work_bytes, void* stream) {
  if (!p || !u4 || !packed || !params || n < 0 || (n > 0 && (!pos || !out)) || (work && work_bytes <= 0))
    return ld_fail(LD_ERR_ARG, "ld_mlp_infer: bad arguments");
  if (p->N > 1024) return ld_fail(LD_ERR_ARG, "ld_mlp_infer: N > 1024 (stencil offsets are 32-bit)");
  if (p->N & (p->N - 1)) return ld_fail(LD_ERR_UNSUPPORTED, "ld_mlp_infer: N = %d (the stencil wrap needs a power of two)", p->N);
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const double L = 2.0 * M_PI;
  static_assert(SMEM_FWD <= 227 * 1024, "tensor-core forward exceeds shared memory");
  // feature tiles and aux live in the caller's workspace, or in the plan's transform workspace
  // (idle during droplet stages that do not overlap the flow's transforms): droplets are taken
  // in batches of whole tiles that fit it
  const size_t per = sizeof(bf16) * K1 + sizeof(float) * 8;
  long long cap = (long long)((work ? (size_t)work_bytes : p->work_bytes) / per);
  cap -= cap % TM;
  if (cap < TM) return ld_fail(LD_ERR_CAPACITY, "ld_mlp_infer: no workspace");
  unsigned char* X = (unsigned char*)(work ? work : p->work);
  for (long long b0 = 0; b0 < n; b0 += cap) {
    const long long nb = n - b0 < cap ? n - b0 : cap;
    const long long tiles = (nb + TM - 1) / TM;
    float* aux = (float*)(X + tiles * (long long)TILE_X_BYTES);
    const long long groups = (nb + FDROP - 1) / FDROP;
    long long gf = (groups + FTHREADS / 32 - 1) / (FTHREADS / 32);
    if (gf > 148LL * 2 * 8) gf = 148LL * 2 * 8;
    const long long gm = tiles < 148 ? tiles : 148;  // one CTA per SM (shared memory, TMEM), persistent
    if (p->prec == LD_F32) {
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_mlp_forward_tc<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)SMEM_FWD));
      {
        ProfScope ps(p, KID_MLP_FEAT, s);
        k_mlp_features<float><<<(unsigned)gf, FTHREADS, 0, s>>>((const float4*)u4, p->N, L,
                                                                          pos + 3 * b0, nb, params, (bf16*)X, aux);
      }
      ProfScope ps(p, KID_MLP_INFER, s);
      k_mlp_forward_tc<float><<<(unsigned)gm, FT_THREADS, SMEM_FWD, s>>>(X, aux, nb, (const bf16*)packed, params,
                                                                        (float*)out + 3 * b0, p->status,
                                                                        p->wait_limit, p->wait_stall);
    } else {
      LD_CUDA_CHECK(cudaFuncSetAttribute(k_mlp_forward_tc<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)SMEM_FWD));
      {
        ProfScope ps(p, KID_MLP_FEAT, s);
        k_mlp_features<double><<<(unsigned)gf, FTHREADS, 0, s>>>((const double4*)u4, p->N, L,
                                                                            pos + 3 * b0, nb, params, (bf16*)X, aux);
      }
      ProfScope ps(p, KID_MLP_INFER, s);
      k_mlp_forward_tc<double><<<(unsigned)gm, FT_THREADS, SMEM_FWD, s>>>(X, aux, nb, (const bf16*)packed,
                                                                         params, (double*)out + 3 * b0, p->status,
                                                                         p->wait_limit, p->wait_stall);
    }
    LD_LAUNCH_CHECK();
  }
  return LD_OK;
}

int ld_phase_shift(ld_plan* p, const void* uk, void* out, double sx, double sy, double sz, void* stream) {
  if (!p || !uk || !out) return ld_fail(LD_ERR_ARG, "ld_phase_shift: bad arguments");
  const double dx = 2.0 * M_PI / p->N;
  const long long cs = p->cube_elems();
  cudaStream_t s = (cudaStream_t)stream;
  if (p->prec == LD_F32)
    k_phase_shift<float><<<gridn(3 * cs, 256), 256, 0, s>>>((const float2*)uk, (float2*)out, cs, p->kc, p->My,
                                                             p->Mzp, sx * dx, sy * dx, sz * dx);
  else
    k_phase_shift<double><<<gridn(3 * cs, 256), 256, 0, s>>>((const double2*)uk, (double2*)out, cs, p->kc, p->My,
                                                              p->Mzp, sx * dx, sy * dx, sz * dx);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_mlp_samples(ld_plan* p, const void* u4, const void* ue, const int64_t* idx, int64_t ns, double sx, double sy,
                   double sz, const float* params, void* X, float* T, float* aux, void* stream) {
  if (!p || !u4 || !ue || ns < 0 || (ns > 0 && (!idx || !params || !X || !T || !aux)))
    return ld_fail(LD_ERR_ARG, "ld_mlp_samples: bad arguments");
  if (p->N > 1024) return ld_fail(LD_ERR_ARG, "ld_mlp_samples: N > 1024 (stencil offsets are 32-bit)");
  if (p->N & (p->N - 1)) return ld_fail(LD_ERR_UNSUPPORTED, "ld_mlp_samples: N = %d (the stencil wrap needs a power of two)", p->N);
  if (ns == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const double L = 2.0 * M_PI;
  if (p->prec == LD_F32)
    k_mlp_samples<float><<<gridn(ns, 128), 128, 0, s>>>((const float4*)u4, (const float*)ue, p->N, L,
                                                        (const long long*)idx, ns, sx, sy, sz, params, (bf16*)X, T, aux);
  else
    k_mlp_samples<double><<<gridn(ns, 128), 128, 0, s>>>((const double4*)u4, (const double*)ue, p->N, L,
                                                         (const long long*)idx, ns, sx, sy, sz, params, (bf16*)X, T,
                                                         aux);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_interleave3(ld_plan* p, const void* planar, void* out, void* stream) {
  if (!p || !planar || !out) return ld_fail(LD_ERR_ARG, "ld_interleave3: bad arguments");
  const long long m = (long long)p->N * p->N * p->N;
  cudaStream_t s = (cudaStream_t)stream;
  if (p->prec == LD_F32) k_interleave3<float><<<gridn(m, 256), 256, 0, s>>>((const float*)planar, (float4*)out, m);
  else k_interleave3<double><<<gridn(m, 256), 256, 0, s>>>((const double*)planar, (double4*)out, m);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_gather4(ld_plan* p, const void* u4, const double* pos, int64_t n, int method, void* out, void* stream) {
  if (!p || !u4 || n < 0 || method < 0 || method > 2 || (n > 0 && (!pos || !out)))
    return ld_fail(LD_ERR_ARG, "ld_gather4: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const double L = 2.0 * M_PI;
  const int g = gridn(n, 256);
#define LD_G4(TT, V4, M) k_gather4<TT, M><<<g, 256, 0, s>>>((const V4*)u4, p->N, L, pos, n, (TT*)out)
  if (p->prec == LD_F32) {
    if (method == LD_INTERP_TRILINEAR) LD_G4(float, float4, LD_INTERP_TRILINEAR);
    else if (method == LD_INTERP_TRICUBIC) LD_G4(float, float4, LD_INTERP_TRICUBIC);
    else LD_G4(float, float4, LD_INTERP_COSINE);
  } else {
    if (method == LD_INTERP_TRILINEAR) LD_G4(double, double4, LD_INTERP_TRILINEAR);
    else if (method == LD_INTERP_TRICUBIC) LD_G4(double, double4, LD_INTERP_TRICUBIC);
    else LD_G4(double, double4, LD_INTERP_COSINE);
  }
#undef LD_G4
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_droplet_predict(ld_plan* p, const double* pos, const void* vel, int64_t n, double h, double* xs,
                       void* stream) {
  if (!p || n < 0 || (n > 0 && (!pos || !vel || !xs))) return ld_fail(LD_ERR_ARG, "ld_droplet_predict: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (p->prec == LD_F32) k_droplet_predict<float><<<gridn(3 * n, 256), 256, 0, s>>>(pos, (const float*)vel, n, h, xs);
  else k_droplet_predict<double><<<gridn(3 * n, 256), 256, 0, s>>>(pos, (const double*)vel, n, h, xs);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_droplet_update(ld_plan* p, int stage, const void* up, double* pos, void* vel, const void* tau, void* a1,
                      int64_t n, double h, double g, void* stream) {
  if (!p || (stage != 1 && stage != 2) || n < 0 || (n > 0 && (!up || !pos || !vel || !tau || !a1)))
    return ld_fail(LD_ERR_ARG, "ld_droplet_update: bad arguments");
  if (n == 0) return LD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  ProfScope ps(p, stage == 1 ? KID_DROPLET1 : KID_DROPLET2, s);
  if (p->prec == LD_F32)
    k_droplet_given<float><<<gridn(n, 256), 256, 0, s>>>(stage, (const float*)up, pos, (float*)vel, (const float*)tau,
                                                         (float*)a1, n, h, (float)g);
  else
    k_droplet_given<double><<<gridn(n, 256), 256, 0, s>>>(stage, (const double*)up, pos, (double*)vel,
                                                          (const double*)tau, (double*)a1, n, h, g);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int64_t ld_mlp_partial_floats(int64_t nb) { return ((nb + TBT - 1) / TBT) * (int64_t)(N_PARAMS + 1); }

int ld_mlp_grad(const void* X, const float* T, const float* W, int64_t nb, const float* params, const void* packed,
                float* work, float* grad, float* loss, void* stream) {
  if (!X || !T || nb < 1 || !params || !packed || !work || !grad || !loss)
    return ld_fail(LD_ERR_ARG, "ld_mlp_grad: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nblk = (int)((nb + TBT - 1) / TBT);
  float* gpart = work;
  float* lpart = work + (long long)nblk * N_PARAMS;
  const float inv_norm = 1.f / (float)nb;
  LD_CUDA_CHECK(cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_TRAIN_TC));
  k_mlp_train_tc<<<nblk, TR_THREADS, SMEM_TRAIN_TC, s>>>((const bf16*)X, T, W, nullptr, nb, inv_norm,
                                                        (const bf16*)packed, params, gpart, lpart);
  k_mlp_reduce<<<gridn(N_PARAMS, 256), 256, 0, s>>>(gpart, lpart, nblk, grad, loss, inv_norm);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_mlp_train_epoch(const void* X, const float* T, const float* W, const uint32_t* order, int64_t nbatch,
                       int64_t batch, float* params, void* packed, float* m, float* v, int64_t step0, double lr,
                       double lr_final, int64_t total, float* work, float* loss_acc, void* stream) {
  if (!X || !T || !order || nbatch < 0 || batch < 1 || batch > (1LL << 30) || !params || !packed || !m || !v ||
      step0 < 0 || !(lr > 0.0) || total < 1 || !work || !loss_acc)
    return ld_fail(LD_ERR_ARG, "ld_mlp_train_epoch: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nblk = (int)((batch + TBT - 1) / TBT);
  float* gpart = work;
  float* lpart = work + (long long)nblk * N_PARAMS;
  const float inv_norm = 1.f / (float)batch;
  const float b1 = 0.9f, b2 = 0.999f;
  LD_CUDA_CHECK(cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_TRAIN_TC));
  for (int64_t b = 0; b < nbatch; ++b) {
    const int64_t k = step0 + b + 1;  // Adam step of this batch
    const double lrk = lr_final > 0.0 ? lr * pow(lr_final / lr, (double)(k < total ? k : total) / (double)total) : lr;
    const float c1 = 1.f - powf(b1, (float)k), c2 = 1.f - powf(b2, (float)k);
    // each launch may begin while the previous one finishes (programmatic dependent launch)
    LD_CUDA_CHECK(launch_pdl(k_mlp_train_tc, nblk, TR_THREADS, SMEM_TRAIN_TC, s, (const bf16*)X, T, W,
                             order + b * batch, (long long)batch, inv_norm, (const bf16*)packed, params, gpart,
                             lpart));
    LD_CUDA_CHECK(launch_pdl(k_mlp_reduce_adam, gridn(OFF_FS, 256), 256, 0, s, (const float*)gpart,
                             (const float*)lpart, nblk, inv_norm, params, m, v, (bf16*)packed, (float)lrk, b1, b2,
                             1e-8f, c1, c2, loss_acc));
  }
  LD_LAUNCH_CHECK();
  return LD_OK;
}

int ld_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t step, float lr, void* packed,
                void* stream) {
  if (!params || !grad || !m || !v || step < 1 || !packed) return ld_fail(LD_ERR_ARG, "ld_mlp_adam: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_mlp_adam<<<gridn(N_PARAMS, 256), 256, 0, s>>>(params, grad, m, v, lr, b1, b2, 1e-8f, c1, c2);
  k_mlp_pack<<<gridn(N_PACKED, 256), 256, 0, s>>>(params, (bf16*)packed);
  LD_LAUNCH_CHECK();
  return LD_OK;
}

}  // extern "C"
