// Internal launch helpers shared by the .cu files of the library.
#pragma once
#include <cuda_runtime.h>

#include "../../include/newton_b200.h"

#define NB_COLLIDE_THREADS 256
#define NB_STEP_THREADS 256

size_t nb_collide_smem_bytes(const NbModelDesc* m);
size_t nb_collide_static_smem_bytes();
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
