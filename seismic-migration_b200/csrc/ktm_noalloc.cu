// ktm_noalloc.cu -- ktmMigratePackedNoAlloc: the fast migration without any
// device allocation, for callers that cannot allocate device memory while they
// run (a processing loop that must never let cudaMalloc / cudaFree synchronise
// the device, or a host framework that has already divided the GPU's memory
// among its own pools and allows no allocation behind its back).
//
// The one scratch buffer of the fast path -- the partial images of the trace
// slices that are summed in a fixed order -- lives in a file-scope device
// array of kNoAllocScratchFloats floats (16 MiB) that every GPU which loads the
// library keeps until the process exits.  Host code only ever sees the array's
// host-side stand-in symbol; its device address is looked up once per device
// with cudaGetSymbolAddress, with that device current, on the first call made
// on that device.  With CUDA's lazy module loading (the default) that lookup is
// also what loads this file's module, which creates the array on the device:
// a one-time implicit allocation at the first call per device, so that call
// belongs in the caller's set-up.
#include "ktm_internal.cuh"

#include <mutex>

namespace ktm {
namespace {

// 4 Mi floats = 16 MiB: up to four partial images of 1 Mi samples, or two of 2 Mi.
constexpr size_t kNoAllocScratchFloats = size_t(4) << 20;
// Largest image: two partial images must fit, or slicing would not be possible.
constexpr size_t kNoAllocMaxImage = kNoAllocScratchFloats / 2;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_noallocScratch[kNoAllocScratchFloats];

std::mutex g_mu;
void* g_scratchPtr[kMaxDevices] = {};

int scratch_for_current_device(void** out)
{
    int dev = 0;
    KTM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(KTM_ERR_LIMIT, "ktmMigratePackedNoAlloc: device ordinal %d >= %d", dev,
                         kMaxDevices);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratchPtr[dev]) {
        void* p = nullptr;
        // the device current now is `dev`: the address is that device's copy
        cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess || p == nullptr)
            return set_error(KTM_ERR_CUDA, "ktmMigratePackedNoAlloc: cudaGetSymbolAddress: %s",
                             cudaGetErrorString(e));
        g_scratchPtr[dev] = p;
    }
    *out = g_scratchPtr[dev];
    return KTM_OK;
}

}  // namespace
}  // namespace ktm

extern "C" int ktmMigratePackedNoAlloc(const ktm_job* j)
{
    using namespace ktm;
    if (!j) return set_error(KTM_ERR_ARG, "NULL job");
    if (!j->deviceMemory || j->mode != KTM_MODE_FAST || !j->tracesPacked)
        return set_error(KTM_ERR_ARG, "ktmMigratePackedNoAlloc takes FAST mode, device memory and a "
                                      "packed trace set (ktmPrepareTraces)");
    // the same checks and arguments as the batched and tuned launches of packed sets
    // (KTM_WEIGHT_PREFOLD with prefolded samples included)
    FastArgs a;
    int rc = packed_args(j, &a);
    if (rc) return rc;
    const size_t nimg = (size_t)a.g.nx * a.g.ny * a.g.nz;
    if (nimg > kNoAllocMaxImage)
        return set_error(KTM_ERR_LIMIT,
                         "ktmMigratePackedNoAlloc: image of %zu samples exceeds the limit of %zu "
                         "(static scratch of %zu floats holds at least two partial images)",
                         nimg, kNoAllocMaxImage, kNoAllocScratchFloats);

    void* scratch = nullptr;
    rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    // every partial image is written completely before the ordered sum reads it,
    // so nothing in the shared array needs clearing between calls
    a.scratch = scratch;
    a.scratchBytes = kNoAllocScratchFloats * sizeof(float);
    // as many trace slices as fit in the array (at most 64): the launch then takes
    // its partial images from the array and allocates nothing
    const size_t maxSlices = nimg > 0 ? kNoAllocScratchFloats / nimg : 1;
    a.slices = (int)(maxSlices < 64 ? maxSlices : 64);
    rc = launch_fast(a, static_cast<cudaStream_t>(j->stream));
    return rc ? rc : set_ok();
}
