/*
 * lucky-droplets B200: C ABI of the forced pseudospectral DNS step with droplets.
 *
 * The reference (Rajarshi-prime/lucky-droplets) is a pair of Python scripts with no FFI; the
 * entry points below replace its Python functions one for one, with plain pointers and sizes.
 * Citations are file:line in the reference (forced-dns-sm.py = F, particles.py = P).
 *
 * Conventions
 *  - Every pointer is a device pointer unless its name ends in _host.  The caller owns every
 *    buffer; a plan owns only its twiddle tables, operator tables and transform workspace.
 *  - `stream` is a cudaStream_t passed as void* (0 = legacy default stream).  No call
 *    synchronises the host except ld_status() and the *_host copies it documents.
 *  - Return value: LD_OK (0) or a negative LD_ERR_*.  ld_last_error() describes the last failure
 *    of the calling thread.  A plan is not thread-safe: use one plan per stream.
 *  - Precision of a plan: LD_F32 (float / complex float) or LD_F64 (double / complex double);
 *    droplet positions are double in both.
 *
 * Spectral layouts (complex, kz fastest):
 *  - reference layout "full": (N, N, N/2+1) indexed (kx, ky, kz) with kx, ky in FFT order, exactly
 *    the array rfft_mpi returns on one rank (F:201-206, F:158);
 *  - "cube": the dealiased cube (Mx, My, Mzp) with Mx = My = 2 kc + 1, kc = floor(N/3),
 *    kx, ky in [-kc, kc] stored 0..kc then -kc..-1, kz in [0, kc] padded with zeros to Mzp (a
 *    multiple of 8).  Every mode the spherical mask of F:129 keeps lies in the cube.
 * Physical layout: (N, N, N) real indexed (x, y, z), z fastest, as u[c] of F:150.
 */
#ifndef LUCKY_DROPLETS_LD_H
#define LUCKY_DROPLETS_LD_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LD_API __attribute__((visibility("default")))
#else
#define LD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define LD_OK 0
#define LD_ERR_ARG (-1)
#define LD_ERR_CUDA (-2)
#define LD_ERR_UNSUPPORTED (-3)
#define LD_ERR_CAPACITY (-4)
#define LD_ERR_NOMEM (-5)

#define LD_F32 0
#define LD_F64 1

/* Device status word bits (ld_status). */
#define LD_STATUS_NONFINITE 1u     /* NaN/Inf met in the state                          */
#define LD_STATUS_BLOWUP 2u        /* max Re(uk) > 100 N^3, the abort test of F:618-620  */
#define LD_STATUS_PAIR_OVERFLOW 4u /* collision pair list exceeded its capacity          */
#define LD_STATUS_WAIT_TIMEOUT 8u  /* a bounded device wait gave up                      */

/* Droplet interpolation kernels. */
#define LD_INTERP_TRILINEAR 0
#define LD_INTERP_TRICUBIC 1   /* tensor-product 4-point Lagrange on offsets -1..2          */
#define LD_INTERP_COSINE 2     /* (1 + cos(pi r / 2dx)) / 4 on offsets -1..2, P:6-20, P:435-511 */

typedef struct ld_plan ld_plan;
typedef struct ld_collider ld_collider;

/* Flow parameters of one time step. */
typedef struct ld_flow_params {
  double dt;        /* time step h (F:29, F:559)                                     */
  double nu;        /* kinematic viscosity (F:83)                                    */
  double f0;        /* power injected per forced shell (F:97)                        */
  int32_t kf_lo;    /* first forced shell (F:90: shell_no = 1..nshells)              */
  int32_t kf_hi;    /* last forced shell                                             */
} ld_flow_params;

/* ---- library ------------------------------------------------------------------------- */
LD_API int ld_version(void);
LD_API const char* ld_last_error(void);

/* ---- plans: grid and spectral operators of F:49-141 ---------------------------------- */
/* Builds the twiddle tables (FP64, rounded once to the plan precision), operator tables and
 * transform workspace for an N^3 grid: N a power of two in [16, 512], or one of the mixed-radix
 * sizes 96, 192, 360, 384 (radix-3 and radix-5 stages; the reference takes any N its slabs
 * divide, F:27-29, F:52-57).  The learned interpolation (ld_mlp_infer, ld_mlp_samples) needs a
 * power of two. */
LD_API int ld_plan_create(ld_plan** plan, int n, int precision);
/* A plan for nbox independent boxes of the same grid (no counterpart in the reference, which runs
 * one box per job): every stage call (ld_rk2if_stage, ld_rk4_stage, ld_velocity_rhs,
 * ld_step_epilogue_plane0) then advances all boxes, each pass one launch over all of them, on
 * states laid out (nbox, 3, Mx, My, Mzp) with physical velocities (nbox, N, N, N, 4); the forcing
 * factors are per box.  The transform workspace grows with nbox.  nbox = 1 is ld_plan_create. */
LD_API int ld_plan_create_boxes(ld_plan** plan, int n, int precision, int nbox);
LD_API int ld_plan_boxes(const ld_plan* plan, int32_t* nbox);
LD_API int ld_plan_destroy(ld_plan* plan);
/* dims[0..7] = N, kc, Mx, My, Mz, Mzp, Nf, precision; work_bytes = transform workspace. */
LD_API int ld_plan_dims(const ld_plan* plan, int32_t* dims, size_t* work_bytes);

/* ---- transforms, F:201-213 ---------------------------------------------------------- */
/* rfft_mpi (F:201-206) on one GPU: ncomp real (N,N,N) fields -> ncomp full-layout spectra,
 * unnormalised forward transform (scipy.fft convention). */
LD_API int ld_rfft_mpi(ld_plan* plan, const void* u, void* fu, int ncomp, void* stream);
/* irfft_mpi (F:208-213): full-layout spectra -> real fields, 1/N^3 normalisation; the imaginary
 * parts of the kz = 0 and kz = N/2 coefficients are ignored, as pocketfft's c2r does. */
LD_API int ld_irfft_mpi(ld_plan* plan, const void* fu, void* u, int ncomp, void* stream);
/* irfft_mpi without any allocation - no counterpart in the reference.  For callers that must not
 * allocate device memory: host frameworks that hand out all device memory from their own pool
 * and forbid driver allocations, and time-critical loops that may not allocate after set-up (an
 * allocation can synchronise the device, take unbounded time or fail mid-run).  No plan: the
 * scratch is a file-scope device array sized for N <= 64 (64*64*33 complex floats, 1.08 MB, held
 * by every GPU that loads the library until the process exits) plus static twiddle tables.  FP32
 * only, N in {16, 32, 64}; larger N returns LD_ERR_UNSUPPORTED.  fu (ncomp, N, N, N/2+1) complex
 * float, u (ncomp, N, N, N) float.  The first call on a device sets that device up (symbol-address
 * lookup and a synchronous twiddle copy) and the first call for each N launches that size's
 * kernels for the first time, so make those first calls before any stream capture.  Calls share
 * the scratch: calls that overlap on the GPU race. */
LD_API int ld_irfft_mpi_noalloc(int n, const void* fu, void* u, int ncomp, void* stream);
/* Dealiased transforms in the cube layout: the same transforms restricted to the modes of the
 * spherical mask (F:129) - the form every transform of the DNS step takes. */
LD_API int ld_irfft_cube(ld_plan* plan, const void* uk, void* u, int ncomp, void* stream);
LD_API int ld_rfft_cube(ld_plan* plan, const void* u, void* uk, int ncomp, void* stream);
/* full -> cube: dealias * full (F:567-569 applies dealias after rfft_mpi); cube -> full. */
LD_API int ld_spec_to_cube(ld_plan* plan, const void* full, void* cube, int ncomp, void* stream);
LD_API int ld_spec_from_cube(ld_plan* plan, const void* cube, void* full, int ncomp, void* stream);
/* The dealiased part of a reference-layout spectrum moved by strided copies, for host state that
 * stays in the reference's layout (F:158) - host (pinned) or device memory on the full side:
 *   direction 0: full (ncomp, N, N, N/2+1) -> cube: the rows kz = 0..kc of every (kx, ky) of the
 *                cube are copied, then the modes outside the mask are zeroed (= ld_spec_to_cube);
 *   direction 1: cube -> full: the same rows are written; no other element of `full` is touched
 *                (they stay whatever they were - zeros for a dealiased state).
 * Four cudaMemcpy3DAsync per component and direction; no counterpart in the reference. */
LD_API int ld_spec_copy_region(ld_plan* plan, const void* src, void* dst, int ncomp, int direction, void* stream);

/* ---- spectrum and forcing, F:232-275 ------------------------------------------------- */
/* Shell energy spectrum e3d_to_e1d(0.5 |uk|^2 normalize) (F:232-233, F:243-245) of a cube-layout
 * 3-vector, FP64, ek[0..N/2] (modes with |k| > N/2 + 1/2 are not counted, as np.histogram drops
 * them).  Deterministic: fixed-order FP64 reduction. */
LD_API int ld_shell_spectrum(ld_plan* plan, const void* uk, double* ek, void* stream);
/* Shell sums (Nf doubles) of Re(conj(a) . b) * normalize over the cube-layout 3-vectors a, b: with
 * b the inviscid, unforced RHS of a this is the transfer behind Pik of save() (F:425-428); the
 * flux spectrum is its reversed cumulative sum (F:428). */
LD_API int ld_shell_cross(ld_plan* plan, const void* a, const void* b, double* out, void* stream);
/* Spectral divergence i k . uk of a cube-layout 3-vector into one cube component (F:216-230; the
 * physical divergence whose maximum save() prints at F:472 is its inverse transform). */
LD_API int ld_divergence_spec(ld_plan* plan, const void* uk, void* divk, void* stream);

/* ---- flow right-hand side, F:287-316 -------------------------------------------------- */
/* ku = P[(u x omega)^ + f] * dealias - visc * nu k^2 uk for a cube-layout 3-vector uk, with
 * the constant-power forcing f of F:239-275 on shells kf_lo..kf_hi (f0 = 0 switches it off).
 * If u_out is not NULL the physical velocity (3, N, N, N) is written too. */
LD_API int ld_velocity_rhs(ld_plan* plan, const void* uk, void* ku, void* u_out,
                    const ld_flow_params* prm, double visc, void* stream);

/* ---- time integration ----------------------------------------------------------------- */
/* RK2 (Heun) with viscous integrating factor E = exp(-nu k^2 h), one stage per call:
 *   stage 1: N1 = N(uk);    ustar = E (uk + h N1);  acc = E (uk + h/2 N1)
 *   stage 2: N2 = N(ustar); uk = acc + h/2 N2
 * N is the RHS above without the viscous term.  u_out (nullable) receives the physical
 * velocity of the stage input (uk at stage 1, ustar at stage 2) for the droplet stages,
 * interleaved (N, N, N, 4) as (u, v, w, 0) per grid point. */
LD_API int ld_rk2if_stage(ld_plan* plan, int stage, void* uk, void* ustar, void* acc, void* u_out,
                   const ld_flow_params* prm, void* stream);
/* Builds on `stream` the tables a time step with these parameters reads (the integrating factor
 * exp(-nu k^2 dt) of ld_rk2if_stage; no counterpart in the reference, whose loop recomputes its
 * operators each step, F:561-562).  ld_rk2if_stage builds it itself when nu dt changes, but a
 * stage captured into a CUDA graph records the build into the graph and leaves the table
 * unmarked; call this before capturing so that captured steps find it built. */
LD_API int ld_plan_prepare(ld_plan* plan, const ld_flow_params* prm, void* stream);
/* Classical RK4 with explicit viscosity, one stage per call (F:335-362):
 *   stage s evaluates ku_s = RHS(y_s) with y_1 = uk and
 *   s=1: acc = uk + h/6 ku1, y = uk + h/2 ku1;  s=2: acc += h/3 ku2, y = uk + h/2 ku2;
 *   s=3: acc += h/3 ku3, y = uk + h ku3;        s=4: uk = acc + h/6 ku4.
 * u_out (nullable) receives the physical velocity of y_s, interleaved (N, N, N, 4). */
LD_API int ld_rk4_stage(ld_plan* plan, int stage, void* uk, void* y, void* acc, void* u_out,
                 const ld_flow_params* prm, void* stream);
/* End of a time step, F:596-620: the irfft->rfft "reality" round trip (which symmetrises the
 * kz = 0 plane: uk(k) <- (uk(k) + conj uk(-k)) / 2), the div-free projection, and the blow-up
 * and NaN test, which raises LD_STATUS_BLOWUP / LD_STATUS_NONFINITE in the status word. */
/* Autotuner of the plan's strided-row (y) transform passes (no counterpart in the reference):
 * times each launch variant on the plan's workspace - ms[8] = [inverse, forward] x [one-shot
 * tiles, pipelined with 1, 2, 3 CTAs per SM] (-1: not available) - and keeps the fastest;
 * choice[2] receives it (0 one-shot, k pipelined with k CTAs per SM).  Synchronises the stream.
 * ld_plan_set_tuning applies a choice found on another plan of the same N and precision. */
LD_API int ld_plan_autotune(ld_plan* plan, double* ms, int32_t* choice, void* stream);
LD_API int ld_plan_set_tuning(ld_plan* plan, const int32_t* choice);
/* Bounded device waits (no counterpart in the reference, whose failures end in comm.Abort,
 * F:618-620): the waits of the plan's pipelined kernels (the fused z pass at N >= 256, the
 * tensor-core MLP forward) give up after `limit` polls (0: the default, 2^24), raise
 * LD_STATUS_WAIT_TIMEOUT, let the copies and MMAs they issued complete, free their tensor memory
 * and return; the launch and the context stay usable.  stall != 0 tests that path: the first wait
 * of every warp (z pass) or warp group (MLP forward) is on a barrier that nothing completes, so
 * it runs out after `limit` polls while the first copy is in flight.  stall = 0 for production. */
LD_API int ld_plan_set_wait_limit(ld_plan* plan, uint32_t limit, int stall);
/* While vk is set (a cube-layout 3-vector), every RHS evaluation of the plan (ld_velocity_rhs,
 * ld_rk4_stage, ld_rk2if_stage) also writes the spectrum of the small-droplet (slow-manifold)
 * velocity of its stage input, v = u - tps Du/Dt - tps g z with Du/Dt = -grad p + nu lap u
 * (F:319-321); vk = NULL switches it off. */
LD_API int ld_slow_manifold(ld_plan* plan, void* vk, double tps, double g);
LD_API int ld_step_epilogue(ld_plan* plan, void* uk, void* stream);
/* The same epilogue restricted to the kz = 0 plane (its reality symmetrisation, projection and
 * checks, F:596-620): the last stage of ld_rk2if_stage (stage 2) and of ld_rk4_stage (stage 4)
 * already applies the epilogue's projection and checks to the kz > 0 modes it writes, so after
 * those stages this call completes the step epilogue (ld_step_epilogue there is also correct: it
 * projects the kz > 0 modes a second time). */
LD_API int ld_step_epilogue_plane0(ld_plan* plan, void* uk, void* stream);

/* ---- whole steps: the body of the time loop, F:571-623 ---------------------------------- */
/* State of ld_step / ld_ensemble_step: caller-owned device buffers. */
typedef struct ld_step_state {
  void* uk;            /* (nbox, 3, Mx, My, Mzp) cube spectrum, advanced in place               */
  void* ustar;         /* the same shape: RK2 stage scratch                                       */
  void* acc;           /* the same shape: RK2 accumulator                                         */
  void* u4;            /* (nbox, N, N, N, 4) physical velocity the droplet stages read            */
  int64_t n;           /* droplets (0: flow only)                                                  */
  double* pos;         /* (n, 3) FP64 positions                                                    */
  void* vel;           /* (n, 3) velocities, plan precision                                        */
  void* tau;           /* (n) Stokes times, plan precision                                         */
  void* a1;            /* (n, 3) Heun stage scratch, plan precision                                */
  double* radius;      /* (n) radii (collisions; nullable without them)                            */
  int64_t* ids;        /* (n) droplet ids, permuted with the droplets (nullable)                   */
  int32_t* box;        /* (n) box of each droplet: ld_ensemble_step; NULL for ld_step              */
  int32_t method;      /* LD_INTERP_*                                                              */
  double g;            /* settling acceleration along -z                                           */
  int32_t sort_every;  /* re-sort into cell order every that many steps (0: never)                 */
  uint32_t* order;     /* (n) permutation scratch of the re-sort                                   */
  void* scratch;       /* n * 24 bytes of row scratch for the re-sort                              */
  int32_t* pairs;      /* (pair_cap, 2) colliding pairs after every step; NULL: no collisions      */
  int64_t pair_cap;
  int64_t* pair_count; /* device: pairs of the last step                                           */
  int64_t* box_counts; /* device (nbox), nullable: pairs per box                                   */
  int64_t step;        /* steps done; sets the re-sort phase; incremented by every step            */
} ld_step_state;
/* nsteps whole steps of one box: RK2 + integrating factor stages with the droplet Heun stages
 * between them, the plane epilogue (F:596-620), the re-sort every sort_every steps and the
 * collision search - the sequence of the Python stepper, so the same kernels give the same
 * bits.  The replacement of one pass of the reference's loop body (F:582-620) per step. */
LD_API int ld_step(ld_plan* plan, ld_collider* collider, ld_step_state* state, const ld_flow_params* prm,
                   int32_t nsteps, void* stream);
/* The same for every box of a multi-box plan (ld_plan_create_boxes) with a multi-box collider
 * (ld_collider_create_boxes); state->box gives each droplet's box.  No counterpart in the
 * reference (one box per run there). */
LD_API int ld_ensemble_step(ld_plan* plan, ld_collider* collider, ld_step_state* state, const ld_flow_params* prm,
                            int32_t nsteps, void* stream);

/* ---- droplets, P:52-111, P:435-511, P:817-837 ----------------------------------------- */
/* Interpolate ncomp physical fields (ncomp, N, N, N) at n positions (n, 3) double:
 * out (n, ncomp) in the plan precision.  Positions are taken modulo L = 2 pi. */
LD_API int ld_gather(ld_plan* plan, const void* field, int ncomp, const double* pos, int64_t n,
              int method, void* out, void* stream);
/* Droplet Heun stage on one flow stage (x' = v, v' = (u(x) - v)/tau - g z; the reference's drag
 * and gravity terms, P:831-834, with tau given per droplet):
 *   stage 1: a1 = (u(x) - v)/tau - g z                                         (writes a1)
 *   stage 2: xs = x + h v, vs = v + h a1, a2 = (u(xs) - vs)/tau - g z,
 *            x <- x + h/2 (v + vs), v <- v + h/2 (a1 + a2)                      (writes x, v)
 * u is the interleaved (N, N, N, 4) velocity the stage functions write; pos (n,3) double, vel (n,3),
 * a1 (n,3) and tau (n) in the plan precision. */
LD_API int ld_droplet_stage(ld_plan* plan, int stage, const void* u, double* pos, void* vel,
                     const void* tau, void* a1, int64_t n, int method, double h, double g,
                     void* stream);
/* The same for the droplets of all boxes of a multi-box plan in one launch: droplet i belongs to
 * box[i] (int32) and samples that box's velocity u + box[i] N^3 (interleaved (nbox, N, N, N, 4)).
 * No counterpart in the reference. */
LD_API int ld_droplet_stage_boxes(ld_plan* plan, int stage, const void* u, const int32_t* box, double* pos,
                                  void* vel, const void* tau, void* a1, int64_t n, int method, double h, double g,
                                  void* stream);

/* ---- exact spectral velocity (no counterpart in the reference) ------------------------- */
/* u_c(x) = (1/N^3) sum_k w_kz Re(uk_c(k) exp(i k.x)) over the modes of the spherical mask of a
 * cube-layout 3-vector uk, in FP64, at n points pos (n,3) double -> out (n,3) double.  This is
 * the continuous extension of irfft_mpi (F:208-213): at grid points the two agree.  Used as the
 * judge of the interpolation error. */
LD_API int ld_exact_sum(ld_plan* plan, const void* uk, const double* pos, int64_t n, double* out, void* stream);

/* ---- learned interpolation (no counterpart in the reference) ------------------------------ */
/* MLP 195 -> 128 SiLU -> 128 SiLU -> 3 on BF16 tensor-core tiles with FP32 accumulation, predicting
 * (exact spectral - tricubic) / (scale * os) from the 4x4x4 stencil of (u, v, w) in an orthonormal
 * polynomial basis, divided by its RMS `scale` and multiplied by per-coefficient feature scales,
 * and the fractional cell offsets minus 1/2.  Parameters: one FP32 vector of n_params (layout,
 * feature scales and output scale os in csrc/ld_mlp.cu); the kernels read a packed BF16 copy
 * (n_packed) made by ld_mlp_pack. */
LD_API int ld_mlp_sizes(int64_t* n_params, int64_t* n_packed, int32_t* k_in, int32_t* batch_tile);
LD_API int ld_mlp_pack(const float* params, void* packed, void* stream);
/* Fused gather + tricubic + MLP at n droplets from the interleaved (N,N,N,4) velocity:
 * out (n,3) = tricubic + scale * os * MLP(features). */
LD_API int ld_mlp_infer(ld_plan* plan, const void* u4, const double* pos, int64_t n, const void* packed,
                        const float* params, void* out, void* stream);
/* The same with the feature tiles in the caller's workspace (work, work_bytes; whole 128-droplet
 * tiles per batch) instead of the plan's transform workspace, so that inference may run on another
 * stream while the plan transforms (the droplet stage overlapping the next flow stage).
 * ld_mlp_infer_workspace_bytes(n) is the size that takes n droplets in one batch. */
LD_API int ld_mlp_infer_ws(ld_plan* plan, const void* u4, const double* pos, int64_t n, const void* packed,
                           const float* params, void* out, void* work, int64_t work_bytes, void* stream);
LD_API int64_t ld_mlp_infer_workspace_bytes(int64_t n);
/* uk * exp(i k.(s dx)) for a cube-layout 3-vector: the field translated so that its grid values are
 * the original field's values at x_j + s dx (s in grid units). */
LD_API int ld_phase_shift(ld_plan* plan, const void* uk, void* out, double sx, double sy, double sz, void* stream);
/* Training samples at grid points idx[i] + s (grid units): X (ns, k_in) bf16 features from the
 * interleaved field u4 with the feature scales of params, T (ns,3) = (exact - tricubic)/(scale * os)
 * with exact = ue (planar (3,N^3), the field phase-shifted by s) at idx[i], aux (ns,4) = tricubic xyz
 * and scale. */
LD_API int ld_mlp_samples(ld_plan* plan, const void* u4, const void* ue, const int64_t* idx, int64_t ns, double sx,
                          double sy, double sz, const float* params, void* X, float* T, float* aux, void* stream);
/* Interpolation of an interleaved (N,N,N,4) velocity at n positions -> out (n,3). */
LD_API int ld_gather4(ld_plan* plan, const void* u4, const double* pos, int64_t n, int method, void* out,
                      void* stream);
/* planar (3, N^3) -> interleaved (N^3, 4) in the plan precision. */
LD_API int ld_interleave3(ld_plan* plan, const void* planar, void* out, void* stream);
/* Heun stage-2 positions xs = pos + h vel (n,3), and the droplet stage of ld_droplet_stage with the
 * fluid velocity at the stage position given in up (n,3) (the learned interpolation supplies it). */
LD_API int ld_droplet_predict(ld_plan* plan, const double* pos, const void* vel, int64_t n, double h, double* xs,
                              void* stream);
LD_API int ld_droplet_update(ld_plan* plan, int stage, const void* up, double* pos, void* vel, const void* tau,
                             void* a1, int64_t n, double h, double g, void* stream);
/* Floats of workspace ld_mlp_grad needs for a batch of nb samples. */
LD_API int64_t ld_mlp_partial_floats(int64_t nb);
/* Weighted mean-squared-error loss sum_r w_r |Y_r - T_r|^2 / nb and its exact gradient over a batch
 * of nb samples (X bf16 (nb, k_in), T (nb,3), W (nb) or null for unit weights): deterministic
 * fixed-order reductions.  grad: n_params floats; loss: 1 float. */
LD_API int ld_mlp_grad(const void* X, const float* T, const float* W, int64_t nb, const float* params,
                       const void* packed, float* work, float* grad, float* loss, void* stream);
/* One epoch of mini-batch training: for batch b = 0 .. nbatch-1, samples order[b*batch ..
 * (b+1)*batch) of X, T, W (as in ld_mlp_grad) give the loss and gradient, then one Adam step
 * (step0 + b + 1, learning rate lr * (lr_final / lr)^(min(step, total) / total), or lr when
 * lr_final <= 0) updates params, m, v and the BF16 copy; *loss_acc += each batch loss.  work:
 * ld_mlp_partial_floats(batch) floats.  Same result as ld_mlp_grad then ld_mlp_adam per batch on
 * the gathered rows.  order holds nbatch * batch row indices of X, T, W, each below their row
 * count (the caller's permutation; the kernels read the rows it names unchecked).  A batch whose
 * kernel gave up a bounded wait adds NaN to *loss_acc. */
LD_API int ld_mlp_train_epoch(const void* X, const float* T, const float* W, const uint32_t* order, int64_t nbatch,
                              int64_t batch, float* params, void* packed, float* m, float* v, int64_t step0,
                              double lr, double lr_final, int64_t total, float* work, float* loss_acc, void* stream);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on the FP32 parameters, then re-packs the BF16 copy. */
LD_API int ld_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t step, float lr, void* packed,
                       void* stream);

/* ---- the reference's droplet physics (F:278-362, P:514-577, P:817-837), FP64 ---------------- */
/* clip_zero of F:278-285 on x (m doubles): out = max(x, 0) * mean(x) / mean(max(x, 0)); with
 * clip_src x itself is clipped too (the reference clips its argument in place).  Deterministic
 * sums; work holds ld_ref_workspace_doubles() doubles. */
LD_API int64_t ld_ref_workspace_doubles(void);
LD_API int ld_clip_zero(double* x, double* out, int64_t m, int clip_src, double* work, void* stream);
/* RK4 bookkeeping of the physical n field and the droplet coordinates (F:341-360):
 * y += a x ; z = x + a y. */
LD_API int ld_axpy(double* y, double a, const double* x, int64_t m, void* stream);
LD_API int ld_waxpy(double* z, const double* x, double a, const double* y, int64_t m, void* stream);
/* n-field RHS pieces (F:325-330): nv = n v (planar 3 x N^3), and on the cube
 * knk = -i k . nvk - fck (the spectra of n v and of the deposited sink fc). */
LD_API int ld_n_products(ld_plan* plan, const double* n, const double* v, double* nv, void* stream);
LD_API int ld_n_combine(ld_plan* plan, const void* nvk, const void* fck, void* knk, void* stream);
/* pRHS of P:817-837 for coord (n, 7) = (x, v, m) with the cosine-interpolated fluid velocity iu,
 * slow-manifold velocity iv (n, 3) and number density ic (n): kp (n, 7) = (v, (u - v)/(St tau_eta)
 * - g z, mdot), mdot (n) = growthfactor (1 + sqrt(st_s/St))^2 n |v - v_slow|, St = (m/factor)^(2/3). */
LD_API int ld_prhs_ref(const double* coord, const double* iu, const double* iv, const double* ic, int64_t n,
                       double factor, double growthfactor, double st_s, double tau_eta, double g, double* kp,
                       double* mdot, void* stream);
/* Positions (n, 3) of the droplet coordinates (n, 7). */
LD_API int ld_extract_pos(const double* coord, int64_t n, double* pos, void* stream);
/* Deposition of mdot with the cosine kernel (exterp_cosine_scalar, P:514-577), deterministic:
 * ld_cell_weights gives each droplet its grid cell (key, with val = index) and its 12 weights;
 * after a stable sort of (key, val) (ld_radix_sort_u32) and ld_cell_starts (N^3 + 1 starts),
 * ld_deposit_pull sums, per grid cell, mdot wx wy wz / dx^3 in the reference's order. */
LD_API int ld_cell_weights(const double* coord, int64_t n, int N, double L, uint32_t* key, uint32_t* val, double* w,
                           void* stream);
LD_API int ld_cell_starts(const uint32_t* skey, int64_t n, int64_t ncell, int32_t* cs, void* stream);
LD_API int ld_deposit_pull(const uint32_t* sval, const int32_t* cs, const double* w, const double* mdot, int N,
                           double L, double* fc, void* stream);

/* ---- collisions (no counterpart in the reference: droplets there never collide) ----------- */
/* A collider owns the workspace of the cell-list search for up to nmax droplets on an
 * nc x nc x nc cell grid (nc = floor(L / cell_size), nc >= 1).  Any cell size gives the same
 * pairs: with nc >= 3, a droplet whose diameter exceeds the cell width L / nc also searches the
 * cells within its diameter (its partners with ri + rj > L / nc), so cells narrower than the
 * largest diameter cut the candidates of a wide radius distribution. */
LD_API int ld_collider_create(ld_collider** collider, int64_t nmax, int32_t nc);
/* A collider for the droplets of nbox independent boxes (each an nc^3 cell grid of the same side
 * L; no counterpart in the reference): cells are keyed box-major, so one sort and one search
 * cover every box and pairs never cross boxes.  Use ld_collide_boxes / ld_cell_order_boxes. */
LD_API int ld_collider_create_boxes(ld_collider** collider, int64_t nmax, int32_t nc, int32_t nbox);
LD_API int ld_collider_destroy(ld_collider* collider);
/* Colliding pairs of n droplets, pos (n,3) double, radius (n) double, in a periodic box of side L:
 * wrapped positions, cell = min(int(p / (L/nc)), nc-1) per axis, minimum-image FP64 distance
 * ((dx*dx + dy*dy) + dz*dz < (ri + rj)^2, no fused multiply-add).  pairs (cap, 2) int32 receive
 * (i, j), i < j, in a deterministic order (by the cell of the pair, with nc >= 3; by i with
 * nc < 3); *count (device int64) receives the number of colliding pairs,
 * which may exceed cap: then only cap pairs are written and LD_STATUS_PAIR_OVERFLOW is raised
 * in the collider's status word (ld_collider_status). */
LD_API int ld_collide(ld_collider* collider, const double* pos, const double* radius, int64_t n, double L,
                      int32_t* pairs, int64_t cap, int64_t* count, void* stream);
/* ld_collide over the droplets of all boxes: droplet i lies in box[i] (int32, < nbox); pairs as
 * ld_collide (array indices; both droplets of a pair in one box), in box order; box_counts
 * (nullable, int64 [nbox], device) receives the pairs of every box. */
LD_API int ld_collide_boxes(ld_collider* collider, const double* pos, const double* radius, const int32_t* box,
                            int64_t n, double L, int32_t* pairs, int64_t cap, int64_t* count, int64_t* box_counts,
                            void* stream);
LD_API int ld_collider_status(ld_collider* collider, uint32_t* flags, int clear, void* stream);
/* Record this collider's launches in the event trace of `plan` (ld_profile); NULL stops. */
LD_API int ld_collider_trace(ld_collider* collider, ld_plan* plan);
/* Device pointers to the cell keys and droplet ids of the last ld_collide call, in cell order
 * (valid until the next call): the order that keeps droplet gathers local. */
LD_API int ld_collider_sorted(ld_collider* collider, const uint32_t** keys, const uint32_t** ids);
/* order[i] = the droplet that comes i-th in cell order (cell key of the wrapped position on the
 * collider's grid, ties by index): the permutation that keeps droplet gathers local in memory. */
LD_API int ld_cell_order(ld_collider* collider, const double* pos, int64_t n, double L, uint32_t* order,
                         void* stream);
/* The same order over the droplets of all boxes (box major, then cell, then index). */
LD_API int ld_cell_order_boxes(ld_collider* collider, const double* pos, const int32_t* box, int64_t n, double L,
                               uint32_t* order, void* stream);
/* dst row i = src row order[i] for n rows of row_bytes bytes (a multiple of 4); src != dst.  Applies
 * a droplet permutation to every per-droplet array (the reference's send(), P:233-275, reorders the
 * droplets the same way and tracks them by prtclid). */
/* Device-to-device copy of `bytes` on the stream (the in-place re-sort copies the permuted rows
 * back, so that the droplet arrays keep their addresses across CUDA-graph replays). */
LD_API int ld_copy_async(void* dst, const void* src, int64_t bytes, void* stream);
LD_API int ld_permute_rows(const void* src, void* dst, const uint32_t* order, int64_t n, int32_t row_bytes,
                           void* stream);
/* Stable LSD radix sort of n (key, value) pairs on the low `bits` bits of the keys, in place,
 * using the collider's workspace (n <= nmax). */
LD_API int ld_radix_sort_u32(ld_collider* collider, uint32_t* keys, uint32_t* values, int64_t n, int bits,
                             void* stream);

/* ---- tracing -------------------------------------------------------------------------- */
/* The reference times only whole steps on the wall clock (F:565-577, F:627).  With tracing on, a
 * plan brackets each of its kernel launches with CUDA events on the launching stream. */
LD_API int ld_profile(ld_plan* plan, int enable);
/* Per kernel id: launches and summed device time (ms) since the last reset; synchronises the
 * recorded events.  Writes up to cap entries and their number to *n_out. */
LD_API int ld_profile_read(ld_plan* plan, int32_t* kid, int64_t* count, double* total_ms, int cap,
                           int32_t* n_out, int reset);
/* Name of a kernel id ("zcross", "xfwd_update", ...), or NULL. */
LD_API const char* ld_kernel_name(int kid);

/* ---- status ------------------------------------------------------------------------- */
/* Reads (and with clear != 0 resets) the plan's device status word.  Synchronises `stream`. */
LD_API int ld_status(ld_plan* plan, uint32_t* flags, int clear, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LUCKY_DROPLETS_LD_H */
