// Internal launch helpers shared by the .cu files of the library.
#pragma once
#include <cuda_runtime.h>

#include "../../include/newton_b200.h"

#define NB_COLLIDE_THREADS 256
#define NB_STEP_THREADS 256

size_t nb_collide_smem_bytes(const NbModelDesc* m);
size_t nb_collide_static_smem_bytes(const NbModelDesc* m);
size_t nb_step_smem_bytes(const NbModelDesc* m);

cudaError_t nb_launch_collide(const NbModelDesc* m, const float* body_q, const NbContactSeg* seg, int grid,
                              cudaStream_t stream);
cudaError_t nb_launch_publish(const NbModelDesc* m, const NbContactSeg* seg, const NbContactsPublic* pub,
                              cudaStream_t stream);
cudaError_t nb_launch_ingest(const NbModelDesc* m, const NbContactsPublic* pub, const NbContactSeg* seg,
                             cudaStream_t stream);
cudaError_t nb_launch_step(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io, const NbContactSeg* seg,
                           float dt, int grid, cudaStream_t stream);
cudaError_t nb_launch_contact_forces(const float* imp, const int32_t* count, int cap, float dt, float* force,
                                     cudaStream_t stream);
int nb_step_slab_words(int compact);
cudaError_t nb_launch_match(const NbModelDesc* m, const float* body_q, const NbContactsPublic* pub,
                            const NbContactSeg* seg, const NbMatchState* st, cudaStream_t stream);
cudaError_t nb_launch_ws_features(const NbModelDesc* m, const float* q, const float* qd,
                                  const NbContactsPublic* pub, const float* prev_lambda, const int32_t* match_index,
                                  int32_t* body_count, float dt, float* feat, cudaStream_t s);
cudaError_t nb_launch_ws_targets(const NbContactsPublic* pub, float* impulse, float* lam, int clear, cudaStream_t s);
cudaError_t nb_launch_ws_infer(const NbWsNet* net, const float* feat, const int32_t* count, int cap, float* out,
                               uint32_t* status, cudaStream_t s);
cudaError_t nb_launch_ws_grads(const NbWsTrain* a, cudaStream_t s);
cudaError_t nb_launch_ws_adam(float* w, const float* g, float* m1, float* m2, long count, float lr, float b1,
                              float b2, float eps, float wd, int step, cudaStream_t s);

// Raises `kernel`'s dynamic shared-memory limit on the current device to at
// least `bytes` (cudaFuncSetAttribute) unless an earlier call on this device
// already did, or the kernel's static shared memory plus `bytes` fits the
// 48 KB a CTA may use without the attribute.  Attributes belong to a device, so the record is kept per
// (kernel, device ordinal); a mutex orders first calls from several host
// threads.  Calls that need no raise touch no attribute, which keeps them
// legal inside CUDA-graph capture.
cudaError_t nb_raise_dynamic_smem(const void* kernel, size_t bytes);

// NB_OK for cudaSuccess; otherwise records e for nb_last_cuda_error() and returns NB_ERR_CUDA
int nb_cuda_rc(cudaError_t e);

cudaError_t nb_launch_xpbd_adjoint(const NbModelDesc* m, const NbXpbdParams* p, const NbAdjointIO* io,
                                   const NbContactSeg* seg, int has_contacts, float dt, cudaStream_t s);

// Grid for grid-stride loops over contact rows: enough blocks of `threads` to
// cover `rows`, at most 8 per SM of the current device.
inline int nb_contact_grid(long rows, int threads = 256) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        sms = 148;
    const long need = (rows + threads - 1) / threads;
    const long cap = 8L * sms;
    return (int)(need < 1 ? 1 : (need < cap ? need : cap));
}
