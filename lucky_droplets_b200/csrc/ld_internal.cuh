// Internal declarations shared by the plan/C-ABI unit and the per-(precision, N) kernel units.
#pragma once
#include <cuda_runtime.h>
#include "ld_common.cuh"

#include <vector>

int ld_fail(int code, const char* fmt, ...);

// Kernel ids of the per-launch event trace (ld_profile / ld_profile_read).
enum LdKernelId : int {
  KID_XINV = 0,      // inverse x pass (with the curl in the DNS step)
  KID_YINV,          // inverse y pass
  KID_ZCROSS,        // fused z pass: C2R, u x w, R2C
  KID_YFWD,          // forward y pass
  KID_XFWD_UPD,      // forward x pass + k-space update
  KID_FORCING,       // forcing-factor shell sums
  KID_EPILOGUE,      // end-of-step symmetrise/project/check
  KID_DROPLET1,      // droplet stage 1
  KID_DROPLET2,      // droplet stage 2
  KID_GATHER,        // standalone interpolation
  KID_ZC2R,          // generic z C2R
  KID_ZR2C,          // generic z R2C
  KID_XPASS,         // generic x pass
  KID_YPASS,         // generic y pass
  KID_CONVERT,       // cube <-> reference layout
  KID_SHELL,         // shell spectrum
  KID_IFAC,          // integrating-factor table
  KID_EXACT,         // exact spectral sum at points
  KID_COLL_SORT,     // collision cell keys + radix sort
  KID_COLL_PAIRS,    // collision ranges, count, scan, emit
  KID_CELL_ORDER,    // droplet cell-order permutation
  KID_MLP_INFER,     // MLP forward of the feature rows (+ tricubic, back to the grid frame)
  KID_MLP_FEAT,      // canonical stencil gather + polynomial features
  KID_COUNT_BASE     // further ids are defined by later units
};

struct ProfRec {
  int kid;
  cudaEvent_t a, b;
};

struct ld_plan {
  int N, kc, Mx, My, Mz, Mzp, Nf, prec;
  int nbox = 1;          // boxes of a multi-box plan (ld_plan_create_boxes): states (nbox, 3, cube)
  size_t esz;            // bytes per real element
  void* tw = nullptr;    // N complex twiddles exp(-2 pi i p / N)
  void* ifac = nullptr;  // exp(-nu h k^2) by k^2 (plan precision)
  int nifac = 0;
  double ifac_key = -1;  // nu*h of the current table
  int* shell_off = nullptr;  // CSR of cube indices per shell
  int* shell_idx = nullptr;
  double* factor = nullptr;  // forcing factor per shell
  unsigned* status = nullptr;
  void* work = nullptr;
  size_t work_bytes = 0;
  void* W1 = nullptr;  // 6 * N * My * Mzp complex
  void* W2 = nullptr;  // 6 * N * N * Mzp complex
  // launch choices of the strided-row (y) passes of the RHS, set by ld_plan_autotune:
  // -1 pipelined with the occupancy-limited grid, 0 one-shot tiles, k > 0 pipelined, k CTAs/SM
  int tune_y[2] = {-1, -1};  // [inverse, forward]
  void* sm_vk = nullptr;          // slow-manifold velocity output of every RHS (none when null)
  double sm_tps = 0.0, sm_g = 0.0;
  unsigned wait_limit = 1u << 24; // polls before a bounded device wait gives up (ld_plan_set_wait_limit)
  int wait_stall = 0;             // test of the time-out path: first waits on a barrier nothing completes
  bool prof = false;              // record per-launch events
  std::vector<ProfRec> recs;      // recorded launches
  std::vector<cudaEvent_t> pool;  // reusable events
  long long cube_elems() const { return (long long)Mx * My * Mzp; }
};


// Bracket a launch with events when tracing is on (stream order: same stream as the launch).
void ld_prof_begin(ld_plan* p, int kid, cudaStream_t s);
void ld_prof_end(ld_plan* p, cudaStream_t s);
struct ProfScope {
  ld_plan* p;
  cudaStream_t s;
  ProfScope(ld_plan* p_, int kid, cudaStream_t s_) : p(p_), s(s_) { if (p && p->prof) ld_prof_begin(p, kid, s); }
  ~ProfScope() { if (p && p->prof) ld_prof_end(p, s); }
};

// Launch sequences of one (precision, N) instance; every pointer is a device pointer.
struct OpsTable {
  int (*rfft_full)(ld_plan*, const void* u, void* fu, int ncomp, cudaStream_t);
  int (*irfft_full)(ld_plan*, const void* fu, void* u, int ncomp, cudaStream_t);
  int (*irfft_cube)(ld_plan*, const void* uk, void* u, int ncomp, cudaStream_t);
  int (*rfft_cube)(ld_plan*, const void* u, void* uk, int ncomp, cudaStream_t);
  int (*to_cube)(ld_plan*, const void* full, void* cube, int ncomp, cudaStream_t);
  int (*from_cube)(ld_plan*, const void* cube, void* full, int ncomp, cudaStream_t);
  int (*shell_spectrum)(ld_plan*, const void* uk, double* ek, cudaStream_t);
  // mode: UpdMode; s0..s3 as documented at k_xfwd_update
  int (*rhs)(ld_plan*, int mode, void* s0, void* s1, void* s2, void* s3, void* uout,
             const ld_flow_params*, double visc, cudaStream_t);
  int (*epilogue)(ld_plan*, void* uk, cudaStream_t);
  int (*epilogue0)(ld_plan*, void* uk, cudaStream_t);
  int (*gather)(ld_plan*, const void* f, int ncomp, const double* pos, long long n, int method, void* out,
                cudaStream_t);
  int (*dstage)(ld_plan*, int stage, int method, const void* u, double* pos, void* vel, const void* tau,
                void* a1, long long n, double h, double g, const int* box, cudaStream_t);
  // times every launch variant of the y passes (ms[2][4]: one-shot, pipelined with 1..3 CTAs/SM)
  // and keeps the fastest in the plan
  int (*autotune)(ld_plan*, cudaStream_t, double* ms);
  // builds the tables a time step of these flow parameters reads (integrating factor)
  int (*prepare)(ld_plan*, const ld_flow_params*, cudaStream_t);
};

// Grid sizes with kernel instances: powers of two 16..512, and the mixed-radix sizes
// 96 = 2^5 3, 192 = 2^6 3, 360 = 2^3 3^2 5 and 384 = 2^7 3 (the grids between 256 and 512 on
// which the FP64 tricubic step is compared at equal interpolation error).
#define LD_FOR_EACH_INSTANCE(X) \
  X(f32, 16) X(f32, 32) X(f32, 64) X(f32, 128) X(f32, 256) X(f32, 512) \
  X(f64, 16) X(f64, 32) X(f64, 64) X(f64, 128) X(f64, 256) X(f64, 512) \
  X(f32, 96) X(f32, 192) X(f32, 360) X(f32, 384) \
  X(f64, 96) X(f64, 192) X(f64, 360) X(f64, 384)
#define LD_DECL_TABLE(P, N) const OpsTable* ops_table_##P##_##N();
LD_FOR_EACH_INSTANCE(LD_DECL_TABLE)
#undef LD_DECL_TABLE
