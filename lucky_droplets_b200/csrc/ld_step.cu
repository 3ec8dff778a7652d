// One-call time stepping: ld_step / ld_ensemble_step advance the flow and its droplets by n whole
// steps - the body of the reference's time loop (F:571-623) with the configuration's RK2 +
// integrating factor, Heun droplets, the re-sort into cell order and the collision search - so
// that a caller from another language needs one entry point per batch of steps.  The sequence is
// the one ForcedDNS._step_one / Ensemble._step_one enqueue (stage 1 of the flow, droplet stage 1,
// stage 2 of the flow, the plane epilogue, droplet stage 2, the re-sort every sort_every steps,
// the collisions); the kernels are the same, so results are bit-identical.
#include "ld_internal.cuh"

extern "C" {

int ld_rk2if_stage(ld_plan* plan, int stage, void* uk, void* ustar, void* acc, void* u_out,
                   const ld_flow_params* prm, void* stream);
int ld_step_epilogue_plane0(ld_plan* plan, void* uk, void* stream);
int ld_droplet_stage(ld_plan* plan, int stage, const void* u, double* pos, void* vel, const void* tau, void* a1,
                     int64_t n, int method, double h, double g, void* stream);
int ld_droplet_stage_boxes(ld_plan* plan, int stage, const void* u, const int32_t* box, double* pos, void* vel,
                           const void* tau, void* a1, int64_t n, int method, double h, double g, void* stream);
int ld_cell_order(ld_collider* collider, const double* pos, int64_t n, double L, uint32_t* order, void* stream);
int ld_cell_order_boxes(ld_collider* collider, const double* pos, const int32_t* box, int64_t n, double L,
                        uint32_t* order, void* stream);
int ld_permute_rows(const void* src, void* dst, const uint32_t* order, int64_t n, int32_t row_bytes, void* stream);
int ld_copy_async(void* dst, const void* src, int64_t bytes, void* stream);
int ld_collide_boxes(ld_collider* collider, const double* pos, const double* radius, const int32_t* box, int64_t n,
                     double L, int32_t* pairs, int64_t cap, int64_t* count, int64_t* box_counts, void* stream);

}  // extern "C"

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

// Re-sort every per-droplet array into the collider's cell order, in place (scratch and copy
// back, so the arrays keep their addresses).
int resort(ld_plan* p, ld_collider* col, ld_step_state* st, void* stream) {
  const int64_t n = st->n;
  if (int rc = st->box ? ld_cell_order_boxes(col, st->pos, st->box, n, kTwoPi, st->order, stream)
                       : ld_cell_order(col, st->pos, n, kTwoPi, st->order, stream))
    return rc;
  const int r = (int)p->esz;
  struct Arr { void* a; int row; };
  const Arr arrs[7] = {{st->pos, 24}, {st->vel, 3 * r}, {st->tau, r}, {st->a1, 3 * r},
                       {st->radius, 8}, {st->ids, 8}, {st->box, 4}};
  for (const Arr& x : arrs) {
    if (!x.a) continue;
    if (int rc = ld_permute_rows(x.a, st->scratch, st->order, n, x.row, stream)) return rc;
    if (int rc = ld_copy_async(x.a, st->scratch, n * (int64_t)x.row, stream)) return rc;
  }
  return LD_OK;
}

int step_n(ld_plan* p, ld_collider* col, ld_step_state* st, const ld_flow_params* prm, int32_t nsteps, void* stream) {
  for (int32_t k = 0; k < nsteps; ++k) {
    const bool drops = st->n > 0;
    if (int rc = ld_rk2if_stage(p, 1, st->uk, st->ustar, st->acc, st->u4, prm, stream)) return rc;
    if (drops) {
      int rc = st->box ? ld_droplet_stage_boxes(p, 1, st->u4, st->box, st->pos, st->vel, st->tau, st->a1, st->n,
                                                st->method, prm->dt, st->g, stream)
                       : ld_droplet_stage(p, 1, st->u4, st->pos, st->vel, st->tau, st->a1, st->n, st->method, prm->dt,
                                          st->g, stream);
      if (rc) return rc;
    }
    if (int rc = ld_rk2if_stage(p, 2, st->uk, st->ustar, st->acc, st->u4, prm, stream)) return rc;
    if (int rc = ld_step_epilogue_plane0(p, st->uk, stream)) return rc;
    if (drops) {
      int rc = st->box ? ld_droplet_stage_boxes(p, 2, st->u4, st->box, st->pos, st->vel, st->tau, st->a1, st->n,
                                                st->method, prm->dt, st->g, stream)
                       : ld_droplet_stage(p, 2, st->u4, st->pos, st->vel, st->tau, st->a1, st->n, st->method, prm->dt,
                                          st->g, stream);
      if (rc) return rc;
    }
    st->step += 1;
    if (drops && st->sort_every > 0 && st->step % st->sort_every == 0)
      if (int rc = resort(p, col, st, stream)) return rc;
    if (drops && st->pairs)
      if (int rc = ld_collide_boxes(col, st->pos, st->radius, st->box, st->n, kTwoPi, st->pairs, st->pair_cap,
                                    st->pair_count, st->box_counts, stream))
        return rc;
  }
  return LD_OK;
}

int check_state(ld_plan* p, ld_collider* col, const ld_step_state* st, const ld_flow_params* prm, int32_t nsteps,
                const char* who) {
  if (!p || !st || !prm || nsteps < 0 || !st->uk || !st->ustar || !st->acc || !st->u4 || st->n < 0)
    return ld_fail(LD_ERR_ARG, "%s: bad arguments", who);
  if (st->n > 0 && (!st->pos || !st->vel || !st->tau || !st->a1 || st->method < 0 || st->method > 2))
    return ld_fail(LD_ERR_ARG, "%s: droplet arrays missing", who);
  if (st->n > 0 && st->sort_every > 0 && (!col || !st->order || !st->scratch))
    return ld_fail(LD_ERR_ARG, "%s: re-sorting needs a collider, order and scratch", who);
  if (st->n > 0 && st->pairs && (!col || !st->radius || !st->pair_count))
    return ld_fail(LD_ERR_ARG, "%s: collisions need a collider, radii and a count", who);
  return LD_OK;
}

}  // namespace

extern "C" {

int ld_step(ld_plan* p, ld_collider* col, ld_step_state* st, const ld_flow_params* prm, int32_t nsteps,
            void* stream) {
  if (int rc = check_state(p, col, st, prm, nsteps, "ld_step")) return rc;
  if (p->nbox != 1 || st->box) return ld_fail(LD_ERR_ARG, "ld_step: one box (use ld_ensemble_step)");
  return step_n(p, col, st, prm, nsteps, stream);
}

int ld_ensemble_step(ld_plan* p, ld_collider* col, ld_step_state* st, const ld_flow_params* prm, int32_t nsteps,
                     void* stream) {
  if (int rc = check_state(p, col, st, prm, nsteps, "ld_ensemble_step")) return rc;
  if (st->n > 0 && !st->box) return ld_fail(LD_ERR_ARG, "ld_ensemble_step: droplet boxes missing");
  return step_n(p, col, st, prm, nsteps, stream);
}

}  // extern "C"
