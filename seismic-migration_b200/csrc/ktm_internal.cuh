// ktm_internal.cuh -- shared declarations of libktm.so (not installed; the
// public ABI is include/ktm.h).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/ktm.h"

namespace ktm {

// ---------------------------------------------------------------- status ---
// Records the status of the calling host thread (ktmGetLastError).
int set_error(int code, const char* fmt, ...);
int set_ok();

#define KTM_CUDA_TRY(expr)                                                      \
    do {                                                                        \
        cudaError_t e_ = (expr);                                                \
        if (e_ != cudaSuccess)                                                  \
            return ::ktm::set_error(e_ == cudaErrorMemoryAllocation             \
                                        ? KTM_ERR_NOMEM : KTM_ERR_CUDA,         \
                                    "%s: %s (%s:%d)", #expr,                    \
                                    cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// ----------------------------------------------------------- kernel args ---
// Image axes and the trace block, as the kernels see them.
struct Geometry {
    int nx, ny, nz;
    float x0, dx, y0, dy, z0, dz;  // axis[i] = start + (float)i * step
    int ntr, nt, stride;           // traces, samples per trace, samples between traces
    float dt;                      // trace sample interval, s
};

// Largest dynamic shared memory a kernel here asks for (B200: 227 KB per CTA).
constexpr int kMaxSmemBytes = 227 * 1024;

// Reference-mode kernel launch (ktm_ref.cu).  All pointers are device memory.
int launch_reference(const Geometry& g, const float* midX, const float* midY,
                     const float* offX, const float* offY, const float* traces,
                     const float* vel, float* image, int accumulate, int tileRun,
                     cudaStream_t stream);

// Fast kernel launch (ktm_fast.cu).  All pointers are device memory.
struct FastArgs {
    Geometry g;
    const float* midX; const float* midY; const float* offX; const float* offY;
    const void* traces; const float* scale; int fmt;
    int pitch;              // elements between traces
    // 0: the kernel evaluates |tau| sqrt(t) per pair (weightMethod says how);
    // 1: sqrt(j*dt) applied to each sample (FP64 device reference only);
    // 2: the packed samples already carry sqrt(j*dt)
    int weightMode;
    int weightMethod;       // KTM_WEIGHT_* when the samples do not carry sqrt(j*dt)
    const float* vel; int velCube;
    float* image; int accumulate;
    int pick; float aperture;
    int tileRun;            // tau samples per warp run (0: chosen from Nz)
    int tileCols;           // image columns per CTA: 24, 12 or 8 (0: 24)
    int chunkCap;           // traces per shared-memory chunk at most (0: as many as fit)
    int slices;             // trace slices (0: chosen to fill the GPU)
    int grad;               // 1: write dI/dv (velocity gradient) instead of the image
    void* scratch;          // optional preallocated partial-image buffer
    size_t scratchBytes;
    unsigned long long* pairsEvaluated;
};
// Fast kernel on a PACKED trace set (ktmPrepareTraces layout); linear pick
// expects samples prefolded with sqrt(j*dt), truncating pick expects them not.
int launch_fast(const FastArgs& a, cudaStream_t stream);

// Persistent batched launch over many jobs (ktm_fast.cu): every job packed, same
// format / pick / weight; images are overwritten.
int launch_batch(const FastArgs* jobs, int njobs, cudaStream_t s);

// Bounded waits of the fast kernels (ktm_fast.cu): how many waits for a chunk's
// bulk copy ran out (the count is reset when read).  Read on stream s after the
// caller's work on s; deviceSync: after all work on the device.
int take_wait_stalls(cudaStream_t s, bool deviceSync, unsigned* n);
// One-CTA self-test of the bulk copy and its bounded wait (stall: wait first on
// a barrier nothing arrives on); checksum = sum of the 64 KiB of 0x01 bytes landed.
int wait_selftest(int stall, unsigned long long limitNs, unsigned* checksum);

// ktm_adjoint.cu: demigration into the packed F32 layout [ntr][pitch]
int launch_demigrate(const Geometry& g, const float* midX, const float* midY, const float* offX,
                     const float* offY, const float* vel, int velCube, const float* image,
                     float* data, int pitch, int pick, int weightMethod, float aperture,
                     int accumulate, cudaStream_t s);

// ktm_api.cu: stream-ordered temporary allocations from the library's own memory
// pool on the current device (release threshold unlimited, so repeated calls
// reuse the memory instead of mapping it again; ktmReleaseMemory trims it).
// Falls back to the device's default pool if a pool cannot be created.
cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t s);

// ktm_api.cu: geometry of a job (validates sizes)
int job_geometry(const ktm_job* j, Geometry* g);
// ktm_api.cu: FastArgs of a device-memory FAST job on a packed trace set (checks the
// job; KTM_WEIGHT_PREFOLD needs tracesPrefolded and becomes weightMode 2)
int packed_args(const ktm_job* j, FastArgs* a);

// ktm_prep.cu
int packed_pitch(int nt, int fmt);
int prepare_traces(const ktm_prep* p);
// F16/BF16 [ntr][stride] (times scale[k] when given) -> new F32 [ntr][nt] buffer
// allocated stream-ordered on s (caller frees with cudaFreeAsync).
int widen_traces(const void* in, int fmt, const float* scale, int ntr, int nt, int stride,
                 void** out, cudaStream_t s);

// ktm_interp.cu: time-axis interpolation by 2^levels (ktmInterpTraces).
int interp_traces(const ktm_interp* p);

// ktm_ibm.cu: IBM-32 words -> IEEE float, bit-identical to ktmIBM32toIEEE.
int ibm_to_ieee(const uint32_t* in, float* out, size_t n, cudaStream_t s);

// FP64 device reference (ktm_fast.cu): out[q][nz] for image columns cols[q]
// (cols == NULL: columns 0..ncols-1).
int launch_f64_columns(const FastArgs& a, const int* cols, int ncols, double* out,
                       cudaStream_t stream);

}  // namespace ktm
