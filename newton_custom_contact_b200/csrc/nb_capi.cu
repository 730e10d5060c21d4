// extern "C" entry points of libnewton_b200.so (declared in include/newton_b200.h).
#include <cuda_runtime.h>

#include <mutex>
#include <utility>
#include <vector>

#include "nb_kernels.cuh"

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_smem_mutex;
// per device: (kernel, dynamic shared-memory bytes already allowed)
std::vector<std::pair<const void*, size_t>> g_smem_raised[kMaxDevices];

int grid_for(int requested) {
    if (requested > 0) return requested;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 2;  // two resident CTAs per SM (__launch_bounds__(256, 2) kernels)
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_model(const NbModelDesc* m) {
    if (!m) return NB_ERR_INVALID;
    if (m->world_count <= 0 || m->body_count < 0 || m->shape_count < 0) return NB_ERR_INVALID;
    if (m->max_world_bodies > 4094) return NB_ERR_UNSUPPORTED;  // 12-bit body tags in contact records
    if (!m->world_body_start || !m->world_joint_start || !m->world_order) return NB_ERR_INVALID;
    if (m->body_count > 0 && (!m->body_com || !m->body_inv_mass || !m->body_inertia || !m->body_inv_inertia ||
                              !m->body_flags || !m->body_world || !m->gravity))
        return NB_ERR_INVALID;
    return NB_OK;
}

int check_seg(const NbContactSeg* s) {
    if (!s || !s->world_count || !s->work_counter || !s->status) return NB_ERR_INVALID;
    if (!s->slots || !s->rec || !s->world_base || !s->cand || !s->cand_count || !s->counts || !s->queue || !s->geom)
        return NB_ERR_INVALID;
    if (!aligned16(s->slots) || !aligned16(s->rec) || !aligned16(s->geom) ||
        (reinterpret_cast<uintptr_t>(s->queue) & 7u) || (reinterpret_cast<uintptr_t>(s->world_base) & 7u))
        return NB_ERR_INVALID;
    return NB_OK;
}

// the step reads only the dense solver records
int check_step_seg(const NbContactSeg* s) {
    if (!s->world_count || !s->world_base || !aligned16(s->rec)) return NB_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(s->world_base) & 7u) return NB_ERR_INVALID;
    return NB_OK;
}

int check_schedule(const NbModelDesc* m) {
    if (m->cta_threads != NB_STEP_THREADS) return NB_ERR_INVALID;
    if (m->smem_floats_per_batch <= 0) return NB_ERR_INVALID;
    if (m->step_mode == 1 || m->step_mode == 2) {
        // independent groups of group_threads: every world's slab must fit one group's share
        const int g = m->group_threads;
        if (g != 32 && g != 64 && g != 128) return NB_ERR_INVALID;
        const int share = (m->smem_floats_per_batch / (NB_STEP_THREADS / g)) & ~1;
        if ((int64_t)m->max_world_bodies * nb_step_slab_words(m->step_mode == 2) > share) return NB_ERR_INVALID;
        if (m->step_mode == 2 && m->body_count > 0 && (!m->body_pack || !aligned16(m->body_pack)))
            return NB_ERR_INVALID;
        return NB_OK;
    }
    if (m->step_mode != 0) return NB_ERR_INVALID;
    const int g = m->group_threads;
    if (g != 32 && g != 64 && g != 128 && g != 256) return NB_ERR_INVALID;
    if (m->batch_count < 0 || (m->batch_count > 0 && (!m->batch_world || !m->batch_slab))) return NB_ERR_INVALID;
    return NB_OK;
}

int smem_limit() {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

}  // namespace

cudaError_t nb_raise_dynamic_smem(const void* kernel, size_t bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_smem_mutex);
    for (auto& kv : g_smem_raised[dev]) {
        if (kv.first != kernel) continue;
        if (bytes <= kv.second) return cudaSuccess;
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e == cudaSuccess) kv.second = bytes;
        return e;
    }
    // without the attribute a CTA may use 48 KB of static and dynamic shared memory together
    cudaFuncAttributes attr;
    e = cudaFuncGetAttributes(&attr, kernel);
    if (e != cudaSuccess) return e;
    const size_t default_limit = attr.sharedSizeBytes < 48 * 1024 ? 48 * 1024 - attr.sharedSizeBytes : 0;
    if (bytes <= default_limit) {
        // within the default limit: nothing to raise, remember that
        g_smem_raised[dev].emplace_back(kernel, default_limit);
        return cudaSuccess;
    }
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) g_smem_raised[dev].emplace_back(kernel, bytes);
    return e;
}

namespace {
// the CUDA error behind the last NB_ERR_CUDA this host thread received
thread_local int g_last_cuda_error = 0;
}  // namespace

int nb_cuda_rc(cudaError_t e) {
    if (e == cudaSuccess) return NB_OK;
    g_last_cuda_error = (int)e;
    return NB_ERR_CUDA;
}

extern "C" {

int nb_abi_version(void) { return NB_ABI_VERSION; }

int nb_last_cuda_error(void) { return g_last_cuda_error; }

const char* nb_cuda_error_string(int code) { return cudaGetErrorString((cudaError_t)code); }

int32_t nb_default_grid(void) { return grid_for(0); }

int nb_clear_forces(float* body_f, int32_t n_bodies, void* stream) {
    if (n_bodies < 0 || (n_bodies > 0 && !body_f)) return NB_ERR_INVALID;
    if (n_bodies == 0) return NB_OK;
    const cudaError_t e = cudaMemsetAsync(body_f, 0, sizeof(float) * 6 * (size_t)n_bodies, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_collide(const NbModelDesc* model, const float* body_q, const NbContactSeg* seg, int32_t grid_ctas,
               void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if ((rc = check_seg(seg))) return rc;
    if (!body_q || !model->world_pair_start || !model->pair_shapes || !model->world_shape_start ||
        (model->global_shape_count > 0 && !model->global_shapes))
        return NB_ERR_INVALID;
    if ((int64_t)(nb_collide_smem_bytes(model) + nb_collide_static_smem_bytes(model)) > smem_limit())
        return NB_ERR_UNSUPPORTED;
    // grid_ctas <= 0: each narrow-phase kernel uses its own default (enough CTAs
    // to reach its register-limited occupancy)
    cudaError_t e = nb_launch_collide(model, body_q, seg, grid_ctas > 0 ? grid_ctas : 0, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_publish_contacts(const NbModelDesc* model, const NbContactSeg* seg, const NbContactsPublic* pub,
                        void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if ((rc = check_seg(seg))) return rc;
    if (!pub || !pub->count || !pub->world_offset || pub->capacity < 0) return NB_ERR_INVALID;
    if (pub->capacity > 0 && (!pub->shape0 || !pub->shape1 || !pub->point0 || !pub->point1 || !pub->offset0 ||
                              !pub->offset1 || !pub->normal || !pub->margin0 || !pub->margin1))
        return NB_ERR_INVALID;
    cudaError_t e = nb_launch_publish(model, seg, pub, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_ingest_contacts(const NbModelDesc* model, const NbContactsPublic* pub, const NbContactSeg* seg,
                       void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if ((rc = check_seg(seg))) return rc;
    if (!pub || !pub->count || pub->capacity < 0) return NB_ERR_INVALID;
    if (!model->world_pair_start || !model->shape_body) return NB_ERR_INVALID;
    cudaError_t e = nb_launch_ingest(model, pub, seg, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_xpbd_step(const NbModelDesc* model, const NbXpbdParams* params, const NbStepIO* io, const NbContactSeg* seg,
                 float dt, int32_t grid_ctas, void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if (!params || !io || !seg || !seg->work_counter || !seg->status) return NB_ERR_INVALID;
    if (params->iterations < 0) return NB_ERR_INVALID;
    if (!(dt > 0.0f)) return NB_ERR_INVALID;
    if (io->contact_impulse && (!io->impulse_scratch || io->contact_impulse_capacity < 0)) return NB_ERR_INVALID;
    if (io->body_parent_f && model->joint_count > 0 && !io->joint_impulse) return NB_ERR_INVALID;
    if (io->ws_lambda && io->ws_capacity < 0) return NB_ERR_INVALID;
    if (params->enable_restitution && seg->rec && !model->shape_restitution) return NB_ERR_INVALID;
    if (model->body_count > 0 && (!io->body_q_in || !io->body_qd_in || !io->body_f_in || !io->body_q_out ||
                                  !io->body_qd_out))
        return NB_ERR_INVALID;
    if ((rc = check_schedule(model))) return rc;
    if (seg->rec && (rc = check_step_seg(seg))) return rc;
    if ((int64_t)nb_step_smem_bytes(model) > smem_limit()) return NB_ERR_UNSUPPORTED;
    cudaError_t e = nb_launch_step(model, params, io, seg, dt, grid_for(grid_ctas), (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_xpbd_step_adjoint(const NbModelDesc* model, const NbXpbdParams* params, const NbAdjointIO* io,
                         const NbContactSeg* seg, float dt, void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if (!params || !io || !seg || !io->status) return NB_ERR_INVALID;
    if (params->iterations < 0 || !(dt > 0.0f)) return NB_ERR_INVALID;
    if (params->enable_restitution) return NB_ERR_UNSUPPORTED;
    if (!model->world_body_start || !model->world_joint_start) return NB_ERR_INVALID;
    const bool forward_only = io->forward_only != 0;
    if (model->body_count > 0 && (!io->body_q_in || !io->body_qd_in || !io->body_f_in || !io->tape_state ||
                                  !io->tape_delta || !io->tape_weight || !io->delta_acc || !io->count_acc))
        return NB_ERR_INVALID;
    if (model->body_count > 0 && !forward_only &&
        (!io->grad_q_out || !io->grad_qd_out || !io->grad_q_in || !io->grad_qd_in || !io->grad_acc))
        return NB_ERR_INVALID;
    if (io->body_q_out && !io->body_qd_out) return NB_ERR_INVALID;
    if (forward_only && !io->body_q_out) return NB_ERR_INVALID;
    const int has_contacts = seg->rec != nullptr && seg->world_count != nullptr && seg->world_base != nullptr;
    if (io->active_capacity < 0 || !io->active_count || (has_contacts && io->active_capacity > 0 && !io->active))
        return NB_ERR_INVALID;
    // replayed branches hold for the forward pass only (the reverse evaluates them at the tape's states)
    if (io->branch_mode < 0 || io->branch_mode > 2 || (io->branch_mode == 2 && !forward_only)) return NB_ERR_INVALID;
    if (io->branch_mode != 0 && (!io->branch_body || (has_contacts && !io->branch_contact))) return NB_ERR_INVALID;
    cudaError_t e = nb_launch_xpbd_adjoint(model, params, io, seg, has_contacts, dt, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_xpbd_substeps(const NbModelDesc* model, const NbXpbdParams* params, const NbStepIO* io,
                     const NbContactSeg* seg, const NbContactsPublic* pub, float dt, int32_t n_substeps,
                     int32_t grid_ctas, void* stream) {
    if (!io || n_substeps < 0) return NB_ERR_INVALID;
    // the plain solve only: per-step outputs (impulses, parent forces) and per-step inputs (warm start)
    // have no meaning across several substeps of one call
    if (io->contact_impulse || io->body_parent_f || io->ws_lambda) return NB_ERR_UNSUPPORTED;
    if (n_substeps == 0) return NB_OK;
    // substep k reads one pair of state buffers and writes the other (the step leaves its input unchanged)
    NbStepIO cur = *io;
    int rc = NB_OK;
    for (int k = 0; k < n_substeps; ++k) {
        const bool odd = (k & 1) != 0;
        cur.body_q_in = odd ? io->body_q_out : io->body_q_in;
        cur.body_qd_in = odd ? io->body_qd_out : io->body_qd_in;
        cur.body_q_out = odd ? const_cast<float*>(io->body_q_in) : io->body_q_out;
        cur.body_qd_out = odd ? const_cast<float*>(io->body_qd_in) : io->body_qd_out;
        if ((rc = nb_collide(model, cur.body_q_in, seg, grid_ctas, stream))) return rc;
        if ((rc = nb_publish_contacts(model, seg, pub, stream))) return rc;
        if ((rc = nb_xpbd_step(model, params, &cur, seg, dt, grid_ctas, stream))) return rc;
    }
    if ((n_substeps & 1) == 0 && model->body_count > 0) {
        // an even count ends in the input buffers: one copy per array into the outputs
        cudaStream_t s = (cudaStream_t)stream;
        if (cudaMemcpyAsync(io->body_q_out, io->body_q_in, sizeof(float) * 7 * (size_t)model->body_count,
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(io->body_qd_out, io->body_qd_in, sizeof(float) * 6 * (size_t)model->body_count,
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return nb_cuda_rc(cudaGetLastError());
    }
    return NB_OK;
}

int nb_match_contacts(const NbModelDesc* model, const float* body_q, const NbContactsPublic* pub,
                      const NbContactSeg* seg, const NbMatchState* st, void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if (!body_q || !pub || !seg || !st || !seg->rec || !model->shape_body) return NB_ERR_INVALID;
    if (!pub->count || !pub->world_offset || !pub->sort_key || pub->capacity != st->capacity) return NB_ERR_INVALID;
    if (st->capacity < 0 || !st->prev_count || !st->prev_world_offset || !st->prev_keys || !st->prev_mid ||
        !st->prev_normal || !st->prev_claim || !st->match_index)
        return NB_ERR_INVALID;
    if (st->sticky && (!st->prev_point0 || !st->prev_point1 || !st->prev_offset0 || !st->prev_offset1 ||
                       !st->prev_normal_sticky))
        return NB_ERR_INVALID;
    if (st->new_indices && (!st->new_count || !st->broken_indices || !st->broken_count || !st->prev_was_matched))
        return NB_ERR_INVALID;
    if (st->capacity == 0) return NB_OK;
    cudaError_t e = nb_launch_match(model, body_q, pub, seg, st, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_ws_features(const NbModelDesc* model, const float* body_q, const float* body_qd, const NbContactsPublic* pub,
                   const float* prev_lambda, const int32_t* match_index, int32_t* body_count, float dt, float* features,
                   void* stream) {
    int rc = check_model(model);
    if (rc) return rc;
    if (!body_q || !body_qd || !pub || !pub->count || !body_count || !features || pub->capacity < 0 ||
        !model->shape_body || !model->shape_mu)
        return NB_ERR_INVALID;
    if (pub->capacity > 0 && (!pub->shape0 || !pub->shape1 || !pub->point0 || !pub->point1 || !pub->normal ||
                              !pub->margin0 || !pub->margin1))
        return NB_ERR_INVALID;
    cudaError_t e = nb_launch_ws_features(model, body_q, body_qd, pub, prev_lambda, match_index, body_count, dt,
                                          features, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_ws_targets(const NbContactsPublic* pub, float* impulse, float* lambda, int32_t clear_impulse, void* stream) {
    if (!pub || !pub->count || !pub->normal || !impulse || !lambda || pub->capacity < 0) return NB_ERR_INVALID;
    cudaError_t e = nb_launch_ws_targets(pub, impulse, lambda, clear_impulse != 0, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_ws_infer(const NbWsNet* net, const float* features, const int32_t* count, int32_t capacity, float* lambda,
                uint32_t* status, void* stream) {
    if (!net || !net->w1 || !net->b1 || !net->w2 || !net->b2 || !net->w3 || !net->b3 || !net->in_mean ||
        !net->in_inv_std || !net->out_scale || !count || !status || capacity < 0)
        return NB_ERR_INVALID;
    if (capacity > 0 && (!features || !lambda)) return NB_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(net->w1) | reinterpret_cast<uintptr_t>(net->w2) |
         reinterpret_cast<uintptr_t>(net->w3)) & 15u)
        return NB_ERR_INVALID;
    cudaError_t e = nb_launch_ws_infer(net, features, count, capacity, lambda, status, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_ws_grads(const NbWsTrain* a, void* stream) {
    if (!a || a->rows <= 0 || !a->x || !a->t || !a->in_mean || !a->in_inv_std || !a->out_scale || !a->w1 ||
        !a->b1 || !a->w2 || !a->b2 || !a->w3 || !a->b3 || !a->g_w1 || !a->g_b1 || !a->g_w2 || !a->g_b2 ||
        !a->g_w3 || !a->g_b3 || !a->xn || !a->z1 || !a->h1 || !a->z2 || !a->h2 || !a->y || !a->dy || !a->dh ||
        !a->dh2 || !a->scratch_wq || !a->loss || !a->status)
        return NB_ERR_INVALID;
    cudaError_t e = nb_launch_ws_grads(a, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_ws_adam(float* w, const float* grad, float* m1, float* m2, int64_t count, float lr, float beta1, float beta2,
               float eps, float weight_decay, int32_t step, void* stream) {
    if (!w || !grad || !m1 || !m2 || count < 0 || step < 1) return NB_ERR_INVALID;
    cudaError_t e = nb_launch_ws_adam(w, grad, m1, m2, (long)count, lr, beta1, beta2, eps, weight_decay, step,
                                      (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

int nb_contact_forces(const float* contact_impulse, const int32_t* count, int32_t capacity, float dt, float* force,
                      void* stream) {
    if (capacity < 0 || (capacity > 0 && (!contact_impulse || !count || !force))) return NB_ERR_INVALID;
    if (!(dt > 0.0f)) return NB_ERR_INVALID;
    cudaError_t e = nb_launch_contact_forces(contact_impulse, count, capacity, dt, force, (cudaStream_t)stream);
    return nb_cuda_rc(e);
}

}  // extern "C"
