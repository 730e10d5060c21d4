// nb_publish_contacts_static: nb_publish_contacts with its scan scratch in a
// file-scope device array instead of a caller buffer.
//
// Who needs it: the reference's Contacts object (newton/_src/sim/contacts.py:43-186)
// owns the dense contact arrays but no per-world offset array, so a foreign
// binding that hands those arrays over as they are has nowhere to put the
// world scan; and hosts that run the publish from a loop where device
// allocation is not allowed (a real-time control loop, or an FFI host that
// has no device allocator of its own) cannot create one on demand.  This
// entry point allocates nothing: no cudaMalloc / cudaFree, no allocating
// library call.
//
// Limits and rules:
//   * model->world_count <= NB_PUBLISH_STATIC_MAX_WORLDS (65536), else
//     NB_ERR_CAPACITY before any device work;
//   * nothing in the scratch has to start at zero: the scan writes all
//     world_count + 1 entries before the publish kernel reads them;
//   * there is one scratch array per device, so calls that can overlap in
//     time on one device (different streams, or host threads that do not
//     order their streams) race on it; calls on one stream are ordered;
//   * the first call on a device looks the array's address up with
//     cudaGetSymbolAddress (which may load the module); make that first call
//     before any stream capture.  The address is cached per device ordinal
//     for the life of the process: a cudaDeviceReset between calls is not
//     supported;
//   * pub->world_offset is neither read nor written, so the per-world
//     offsets that nb_match_contacts reads are not produced here: callers
//     that match contacts use nb_publish_contacts.
#include <cuda_runtime.h>

#include <mutex>

#include "nb_kernels.cuh"

namespace {

constexpr int kMaxDevices = 64;

// scan scratch: world offsets [W+1], 512 KB per device
static __device__ __align__(256) int64_t g_world_offset_scratch[NB_PUBLISH_STATIC_MAX_WORLDS + 1];

std::mutex g_lookup_mutex;
int64_t* g_scratch_ptr[kMaxDevices] = {};

// device address of the scratch array on the current device, looked up once
cudaError_t scratch_address(int64_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_lookup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_world_offset_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<int64_t*>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int nb_publish_contacts_static(const NbModelDesc* model, const NbContactSeg* seg,
                                          const NbContactsPublic* pub, void* stream) {
    if (!model || !seg || !pub) return NB_ERR_INVALID;
    if (model->world_count <= 0) return NB_ERR_INVALID;
    if (model->world_count > NB_PUBLISH_STATIC_MAX_WORLDS) return NB_ERR_CAPACITY;
    int64_t* scratch = nullptr;
    const cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess) return nb_cuda_rc(e);
    NbContactsPublic p = *pub;
    p.world_offset = scratch;
    return nb_publish_contacts(model, seg, &p, stream);
}
