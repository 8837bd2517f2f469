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
// on that device.
#include "ktm_internal.cuh"

#include <cstring>
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
    if (!j->deviceMemory)
        return set_error(KTM_ERR_ARG, "ktmMigratePackedNoAlloc takes device memory only");
    if (j->mode != KTM_MODE_FAST || !j->tracesPacked)
        return set_error(KTM_ERR_ARG, "ktmMigratePackedNoAlloc takes FAST mode and a packed trace "
                                      "set (ktmPrepareTraces)");
    if (j->traceFormat < KTM_FMT_F32 || j->traceFormat > KTM_FMT_BF16)
        return set_error(KTM_ERR_ARG, "bad traceFormat %d", j->traceFormat);
    if (j->pick != KTM_PICK_TRUNCATE && j->pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "bad pick %d", j->pick);
    if (j->weightMethod != KTM_WEIGHT_TABLE && j->weightMethod != KTM_WEIGHT_SQRT)
        return set_error(KTM_ERR_ARG, "bad weightMethod %d", j->weightMethod);
    if (j->imageX.imagePnts < 0 || j->imageY.imagePnts < 0 || j->imageZ.imagePnts < 0 ||
        j->config.traceNo < 0 || j->config.tracePts < 0 || !(j->config.traceSampleRate > 0.0f))
        return set_error(KTM_ERR_ARG, "bad sizes or sample rate");
    const size_t nimg = (size_t)j->imageX.imagePnts * j->imageY.imagePnts * j->imageZ.imagePnts;
    if (nimg > kNoAllocMaxImage)
        return set_error(KTM_ERR_LIMIT,
                         "ktmMigratePackedNoAlloc: image of %zu samples exceeds the limit of %zu "
                         "(static scratch of %zu floats holds at least two partial images)",
                         nimg, kNoAllocMaxImage, kNoAllocScratchFloats);
    if (j->config.traceNo > 0 && (!j->midX || !j->midY || !j->offX || !j->offY || !j->traces ||
                                  !j->traceScale))
        return set_error(KTM_ERR_ARG, "NULL coordinate, trace or scale pointer");
    if (nimg > 0 && (!j->image || !j->velocity)) return set_error(KTM_ERR_ARG, "NULL image or velocity");

    void* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;

    FastArgs a;
    std::memset(&a, 0, sizeof(a));
    Geometry& g = a.g;
    g.nx = j->imageX.imagePnts; g.ny = j->imageY.imagePnts; g.nz = j->imageZ.imagePnts;
    g.x0 = j->imageX.imageStart; g.dx = j->imageX.imageStep;
    g.y0 = j->imageY.imageStart; g.dy = j->imageY.imageStep;
    g.z0 = j->imageZ.imageStart; g.dz = j->imageZ.imageStep;
    g.ntr = j->config.traceNo; g.nt = j->config.tracePts;
    g.stride = j->traceStride > 0 ? j->traceStride : j->config.tracePts;
    g.dt = j->config.traceSampleRate;
    a.midX = j->midX; a.midY = j->midY; a.offX = j->offX; a.offY = j->offY;
    a.traces = j->traces; a.scale = j->traceScale; a.fmt = j->traceFormat; a.pitch = g.stride;
    a.weightMode = j->tracesPrefolded ? 2 : 0;
    a.weightMethod = j->weightMethod;
    a.vel = j->velocity; a.velCube = j->velocityCube;
    a.image = j->image; a.accumulate = j->accumulate;
    a.pick = j->pick; a.aperture = j->aperture;
    a.tileRun = j->tileRun;
    a.pairsEvaluated = j->pairsEvaluated;
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
