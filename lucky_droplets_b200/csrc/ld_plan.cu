// Plans and the extern "C" entry points of include/ld.h.  The launch sequences live in
// ld_ops.cuh and are instantiated per (precision, N) in the ld_inst_*.cu units.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "ld_internal.cuh"
#include "ld_kernels.cuh"

static thread_local char g_last_error[512] = "";

void ld_set_last_error(cudaError_t e) {
  snprintf(g_last_error, sizeof(g_last_error), "CUDA error %d: %s", (int)e, cudaGetErrorString(e));
}

int ld_fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void ld_prof_begin(ld_plan* p, int kid, cudaStream_t s) {
  ProfRec r;
  r.kid = kid;
  for (int i = 0; i < 2; ++i) {
    cudaEvent_t e;
    if (!p->pool.empty()) {
      e = p->pool.back();
      p->pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
      return;
    }
    (i ? r.b : r.a) = e;
  }
  cudaEventRecord(r.a, s);
  p->recs.push_back(r);
}

void ld_prof_end(ld_plan* p, cudaStream_t s) {
  if (!p->recs.empty()) cudaEventRecord(p->recs.back().b, s);
}

static const char* const kKernelNames[] = {
    "xinv", "yinv", "zcross", "yfwd", "xfwd_update", "forcing", "epilogue", "droplet1", "droplet2", "gather",
    "z_c2r", "z_r2c", "xpass", "ypass", "convert", "shell", "ifac", "exact_sum", "collide_sort", "collide_pairs", "cell_order", "mlp_infer", "mlp_features"};

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

const OpsTable* table_of(const ld_plan* p) {
#define LD_PICK(P, NN) \
  if (p->N == NN && ((p->prec == LD_F32) == (std::strcmp(#P, "f32") == 0))) return ops_table_##P##_##NN();
  LD_FOR_EACH_INSTANCE(LD_PICK)
#undef LD_PICK
  return nullptr;
}

int check_plan(const ld_plan* p) {
  if (!p) return ld_fail(LD_ERR_ARG, "null plan");
  return LD_OK;
}

}  // namespace

// =============================================================================================
// extern "C"
// =============================================================================================
extern "C" {

int ld_version(void) { return 1; }

const char* ld_last_error(void) { return g_last_error; }

int ld_plan_create(ld_plan** out, int n, int precision) { return ld_plan_create_boxes(out, n, precision, 1); }

int ld_plan_create_boxes(ld_plan** out, int n, int precision, int nbox) {
  if (!out) return ld_fail(LD_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (nbox < 1 || nbox > 4096) return ld_fail(LD_ERR_ARG, "ld_plan_create_boxes: nbox = %d", nbox);
  if (precision != LD_F32 && precision != LD_F64) return ld_fail(LD_ERR_ARG, "precision %d", precision);
  {
    ld_plan probe;
    probe.N = n;
    probe.prec = precision;
    if (!table_of(&probe))
      return ld_fail(LD_ERR_UNSUPPORTED, "N=%d: grids are powers of two in [16, 512] or 96, 192, 360, 384", n);
  }
  ld_plan* p = new (std::nothrow) ld_plan();
  if (!p) return ld_fail(LD_ERR_NOMEM, "host allocation failed");
  p->N = n;
  p->prec = precision;
  p->nbox = nbox;
  p->esz = precision == LD_F32 ? sizeof(float) : sizeof(double);
  p->kc = n / 3;
  p->Mx = p->My = 2 * p->kc + 1;
  p->Mz = p->kc + 1;
  p->Mzp = (p->Mz + 7) / 8 * 8;
  p->Nf = n / 2 + 1;
  const size_t csz = 2 * p->esz;
  auto cleanup = [&](int rc) { ld_plan_destroy(p); return rc; };
  // twiddles, FP64 then rounded once
  {
    std::vector<double> tw(2 * n);
    for (int i = 0; i < n; ++i) {
      const double a = -2.0 * M_PI * (double)i / (double)n;
      tw[2 * i] = std::cos(a);
      tw[2 * i + 1] = std::sin(a);
    }
    cudaError_t e = cudaMalloc(&p->tw, csz * n);
    if (e != cudaSuccess) { ld_set_last_error(e); return cleanup(LD_ERR_CUDA); }
    if (precision == LD_F32) {
      std::vector<float> tf(2 * n);
      for (int i = 0; i < 2 * n; ++i) tf[i] = (float)tw[i];
      e = cudaMemcpy(p->tw, tf.data(), csz * n, cudaMemcpyHostToDevice);
    } else {
      e = cudaMemcpy(p->tw, tw.data(), csz * n, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) { ld_set_last_error(e); return cleanup(LD_ERR_CUDA); }
  }
  // shell CSR over the cube (histogram bins of F:137-138; |k| > Nf - 1/2 dropped)
  {
    const int kc = p->kc, My = p->My, Mzp = p->Mzp, Nf = p->Nf;
    std::vector<int> cnt(Nf + 1, 0);
    const long long kmax2 = (long long)Nf * Nf - Nf;
    auto shell_of = [&](long long k2) { int s = 0; while ((long long)s * s + s < k2) ++s; return s; };
    std::vector<std::pair<int, int>> items;
    items.reserve((size_t)p->cube_elems());
    for (int ix = 0; ix < My; ++ix)
      for (int iy = 0; iy < My; ++iy)
        for (int kz = 0; kz <= kc; ++kz) {
          const int kx = ix <= kc ? ix : ix - My, ky = iy <= kc ? iy : iy - My;
          const long long k2 = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
          if (k2 > kmax2) continue;
          const int s = shell_of(k2);
          cnt[s + 1]++;
          items.push_back({s, (int)(((long long)ix * My + iy) * Mzp + kz)});
        }
    for (int s = 0; s < Nf; ++s) cnt[s + 1] += cnt[s];
    std::vector<int> idx(items.size());
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    for (auto& it : items) idx[pos[it.first]++] = it.second;
    cudaError_t e = cudaMalloc(&p->shell_off, sizeof(int) * (Nf + 1));
    if (e == cudaSuccess) e = cudaMalloc(&p->shell_idx, sizeof(int) * (idx.size() ? idx.size() : 1));
    if (e == cudaSuccess) e = cudaMemcpy(p->shell_off, cnt.data(), sizeof(int) * (Nf + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && idx.size()) e = cudaMemcpy(p->shell_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->factor, sizeof(double) * Nf * nbox);
    if (e == cudaSuccess) e = cudaMemset(p->factor, 0, sizeof(double) * Nf * nbox);
    if (e == cudaSuccess) e = cudaMalloc(&p->status, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(p->status, 0, sizeof(unsigned));
    p->nifac = 3 * p->kc * p->kc + 1;
    if (e == cudaSuccess) e = cudaMalloc(&p->ifac, p->esz * p->nifac);
    if (e != cudaSuccess) { ld_set_last_error(e); return cleanup(LD_ERR_CUDA); }
  }
  // transform workspace
  {
    const size_t w1 = (size_t)6 * n * p->My * p->Mzp * csz * nbox;
    const size_t w2 = (size_t)6 * n * n * p->Mzp * csz * nbox;
    p->work_bytes = w1 + w2;
    cudaError_t e = cudaMalloc(&p->work, p->work_bytes);
    if (e != cudaSuccess) { ld_set_last_error(e); return cleanup(LD_ERR_CUDA); }
    p->W1 = p->work;
    p->W2 = (char*)p->work + w1;
  }
  *out = p;
  return LD_OK;
}

int ld_plan_destroy(ld_plan* p) {
  if (!p) return LD_OK;
  for (auto& r : p->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  for (auto e : p->pool) cudaEventDestroy(e);
  cudaFree(p->tw);
  cudaFree(p->ifac);
  cudaFree(p->shell_off);
  cudaFree(p->shell_idx);
  cudaFree(p->factor);
  cudaFree(p->status);
  cudaFree(p->work);
  delete p;
  return LD_OK;
}

int ld_plan_boxes(const ld_plan* p, int32_t* nbox) {
  if (int rc = check_plan(p)) return rc;
  if (!nbox) return ld_fail(LD_ERR_ARG, "ld_plan_boxes: bad arguments");
  *nbox = p->nbox;
  return LD_OK;
}

int ld_plan_dims(const ld_plan* p, int32_t* dims, size_t* work_bytes) {
  if (int rc = check_plan(p)) return rc;
  if (dims) {
    dims[0] = p->N; dims[1] = p->kc; dims[2] = p->Mx; dims[3] = p->My;
    dims[4] = p->Mz; dims[5] = p->Mzp; dims[6] = p->Nf; dims[7] = p->prec;
  }
  if (work_bytes) *work_bytes = p->work_bytes;
  return LD_OK;
}

int ld_rfft_mpi(ld_plan* p, const void* u, void* fu, int ncomp, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !fu || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_rfft_mpi: bad arguments");
  return table_of(p)->rfft_full(p, u, fu, ncomp, S(stream));
}

int ld_irfft_mpi(ld_plan* p, const void* fu, void* u, int ncomp, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !fu || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_irfft_mpi: bad arguments");
  return table_of(p)->irfft_full(p, fu, u, ncomp, S(stream));
}

int ld_irfft_cube(ld_plan* p, const void* uk, void* u, int ncomp, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !uk || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_irfft_cube: bad arguments");
  return table_of(p)->irfft_cube(p, uk, u, ncomp, S(stream));
}

int ld_rfft_cube(ld_plan* p, const void* u, void* uk, int ncomp, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !uk || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_rfft_cube: bad arguments");
  return table_of(p)->rfft_cube(p, u, uk, ncomp, S(stream));
}

int ld_spec_to_cube(ld_plan* p, const void* full, void* cube, int ncomp, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!full || !cube || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_spec_to_cube: bad arguments");
  return table_of(p)->to_cube(p, full, cube, ncomp, S(stream));
}

int ld_spec_from_cube(ld_plan* p, const void* cube, void* full, int ncomp, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!full || !cube || ncomp < 1) return ld_fail(LD_ERR_ARG, "ld_spec_from_cube: bad arguments");
  return table_of(p)->from_cube(p, cube, full, ncomp, S(stream));
}

int ld_shell_spectrum(ld_plan* p, const void* uk, double* ek, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!uk || !ek) return ld_fail(LD_ERR_ARG, "ld_shell_spectrum: bad arguments");
  return table_of(p)->shell_spectrum(p, uk, ek, S(stream));
}

int ld_velocity_rhs(ld_plan* p, const void* uk, void* ku, void* u_out, const ld_flow_params* prm, double visc,
                    void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!uk || !ku || !prm) return ld_fail(LD_ERR_ARG, "ld_velocity_rhs: bad arguments");
  if (prm->kf_hi >= p->Nf) return ld_fail(LD_ERR_ARG, "forced shell out of range");
  return table_of(p)->rhs(p, ld::UPD_RHS, ku, (void*)uk, nullptr, nullptr, u_out, prm, visc, S(stream));
}

int ld_rk2if_stage(ld_plan* p, int stage, void* uk, void* ustar, void* acc, void* u_out, const ld_flow_params* prm,
                   void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!uk || !ustar || !acc || !prm || (stage != 1 && stage != 2)) return ld_fail(LD_ERR_ARG, "ld_rk2if_stage: bad arguments");
  if (prm->kf_hi >= p->Nf) return ld_fail(LD_ERR_ARG, "forced shell out of range");
  if (stage == 1) return table_of(p)->rhs(p, ld::UPD_RK2_1, ustar, uk, acc, nullptr, u_out, prm, 0.0, S(stream));
  return table_of(p)->rhs(p, ld::UPD_RK2_2, uk, ustar, acc, nullptr, u_out, prm, 0.0, S(stream));
}

int ld_rk4_stage(ld_plan* p, int stage, void* uk, void* y, void* acc, void* u_out, const ld_flow_params* prm,
                 void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!uk || !y || !acc || !prm || stage < 1 || stage > 4) return ld_fail(LD_ERR_ARG, "ld_rk4_stage: bad arguments");
  if (prm->kf_hi >= p->Nf) return ld_fail(LD_ERR_ARG, "forced shell out of range");
  // stage input: uk at stage 1, y afterwards; the next stage input is written to y
  void* in = stage == 1 ? uk : y;
  return table_of(p)->rhs(p, ld::UPD_RK4_1 + stage - 1, uk, in, acc, y, u_out, prm, 1.0, S(stream));
}

int ld_plan_autotune(ld_plan* p, double* ms, int32_t* choice, void* stream) {
  if (int rc = check_plan(p)) return rc;
  double t[8];
  if (int rc = table_of(p)->autotune(p, S(stream), t)) return rc;
  if (ms)
    for (int i = 0; i < 8; ++i) ms[i] = t[i];
  if (choice) { choice[0] = p->tune_y[0]; choice[1] = p->tune_y[1]; }
  return LD_OK;
}

int ld_plan_set_tuning(ld_plan* p, const int32_t* choice) {
  if (int rc = check_plan(p)) return rc;
  if (!choice || choice[0] < -1 || choice[0] > 3 || choice[1] < -1 || choice[1] > 3)
    return ld_fail(LD_ERR_ARG, "ld_plan_set_tuning: bad arguments");
  p->tune_y[0] = choice[0];
  p->tune_y[1] = choice[1];
  return LD_OK;
}

int ld_plan_prepare(ld_plan* p, const ld_flow_params* prm, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!prm) return ld_fail(LD_ERR_ARG, "ld_plan_prepare: bad arguments");
  return table_of(p)->prepare(p, prm, S(stream));
}

int ld_plan_set_wait_limit(ld_plan* p, uint32_t limit, int stall) {
  if (int rc = check_plan(p)) return rc;
  p->wait_limit = limit == 0 ? (1u << 24) : limit;
  p->wait_stall = stall ? 1 : 0;
  return LD_OK;
}

int ld_slow_manifold(ld_plan* p, void* vk, double tps, double g) {
  if (int rc = check_plan(p)) return rc;
  p->sm_vk = vk;
  p->sm_tps = tps;
  p->sm_g = g;
  return LD_OK;
}

int ld_step_epilogue(ld_plan* p, void* uk, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!uk) return ld_fail(LD_ERR_ARG, "ld_step_epilogue: bad arguments");
  return table_of(p)->epilogue(p, uk, S(stream));
}

int ld_step_epilogue_plane0(ld_plan* p, void* uk, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!uk) return ld_fail(LD_ERR_ARG, "ld_step_epilogue_plane0: bad arguments");
  return table_of(p)->epilogue0(p, uk, S(stream));
}

int ld_gather(ld_plan* p, const void* field, int ncomp, const double* pos, int64_t n, int method, void* out,
              void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!field || !pos || !out || ncomp < 1 || ncomp > 8 || n < 0 || method < 0 || method > 2)
    return ld_fail(LD_ERR_ARG, "ld_gather: bad arguments");
  if (n == 0) return LD_OK;
  return table_of(p)->gather(p, field, ncomp, pos, n, method, out, S(stream));
}

int ld_droplet_stage(ld_plan* p, int stage, const void* u, double* pos, void* vel, const void* tau, void* a1,
                     int64_t n, int method, double h, double g, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !pos || !vel || !tau || !a1 || n < 0 || method < 0 || method > 2 || (stage != 1 && stage != 2))
    return ld_fail(LD_ERR_ARG, "ld_droplet_stage: bad arguments");
  if (n == 0) return LD_OK;
  return table_of(p)->dstage(p, stage, method, u, pos, vel, tau, a1, n, h, g, nullptr, S(stream));
}

int ld_droplet_stage_boxes(ld_plan* p, int stage, const void* u, const int32_t* box, double* pos, void* vel,
                           const void* tau, void* a1, int64_t n, int method, double h, double g, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !box || !pos || !vel || !tau || !a1 || n < 0 || method < 0 || method > 2 || (stage != 1 && stage != 2))
    return ld_fail(LD_ERR_ARG, "ld_droplet_stage_boxes: bad arguments");
  if (n == 0) return LD_OK;
  return table_of(p)->dstage(p, stage, method, u, pos, vel, tau, a1, n, h, g, box, S(stream));
}

int ld_profile(ld_plan* p, int enable) {
  if (int rc = check_plan(p)) return rc;
  p->prof = enable != 0;
  return LD_OK;
}

int ld_profile_read(ld_plan* p, int32_t* kid, int64_t* count, double* total_ms, int cap, int32_t* n_out, int reset) {
  if (int rc = check_plan(p)) return rc;
  const int K = 64;
  std::vector<long long> cnt(K, 0);
  std::vector<double> ms(K, 0.0);
  for (auto& r : p->recs) {
    LD_CUDA_CHECK(cudaEventSynchronize(r.b));
    float t = 0.f;
    LD_CUDA_CHECK(cudaEventElapsedTime(&t, r.a, r.b));
    if (r.kid >= 0 && r.kid < K) { cnt[r.kid]++; ms[r.kid] += t; }
  }
  int n = 0;
  for (int k = 0; k < K; ++k) {
    if (!cnt[k]) continue;
    if (n < cap) {
      if (kid) kid[n] = k;
      if (count) count[n] = cnt[k];
      if (total_ms) total_ms[n] = ms[k];
    }
    ++n;
  }
  if (n_out) *n_out = n;
  if (reset) {
    for (auto& r : p->recs) { p->pool.push_back(r.a); p->pool.push_back(r.b); }
    p->recs.clear();
  }
  return LD_OK;
}

const char* ld_kernel_name(int kid) {
  const int n = (int)(sizeof(kKernelNames) / sizeof(kKernelNames[0]));
  return (kid >= 0 && kid < n) ? kKernelNames[kid] : nullptr;
}

int ld_status(ld_plan* p, uint32_t* flags, int clear, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!flags) return ld_fail(LD_ERR_ARG, "ld_status: null flags");
  unsigned h = 0;
  LD_CUDA_CHECK(cudaMemcpyAsync(&h, p->status, sizeof(unsigned), cudaMemcpyDeviceToHost, S(stream)));
  LD_CUDA_CHECK(cudaStreamSynchronize(S(stream)));
  if (clear) LD_CUDA_CHECK(cudaMemsetAsync(p->status, 0, sizeof(unsigned), S(stream)));
  *flags = h;
  return LD_OK;
}

}  // extern "C"
