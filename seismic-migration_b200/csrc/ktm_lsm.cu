// ktm_lsm.cu -- least-squares migration by CGLS on the device.
//
//   minimise || L m - d ||^2,  L = demigration (ktm_adjoint.cu),
//                              L^T = migration (ktm_fast.cu, packed F32 data)
//   r0 = d - L m0, s0 = L^T r0, p0 = s0, gamma0 = <s0, s0>
//   per iteration: q = L p; alpha = gamma / <q, q>; m += alpha p; r -= alpha q;
//                  s = L^T r; gamma' = <s, s>; beta = gamma'/gamma; p = s + beta p
//
// Vectors are FP32 (data in the packed F32 layout with zero guards, so the
// migration reads the residual directly); dot products, norms and the CG
// scalars are FP64 and never leave the device during the iterations: the
// scalar updates are one-thread kernels reading and writing device memory, so
// one iteration is a fixed launch sequence that is captured once in a CUDA
// graph and replayed.
#include "ktm_internal.cuh"

#include <algorithm>
#include <cstring>

namespace ktm {
namespace {

constexpr int kDotBlocks = 592;        // 4 x 148 SMs
constexpr int kDotThreads = 256;

// scalar slots in the FP64 state array
enum { kGamma = 0, kDelta, kAlpha, kBeta, kGammaNew, kRr, kIter, kNScalars };

__global__ void dot_partial(const float* __restrict__ x, const float* __restrict__ y, size_t n,
                            double* __restrict__ partial)
{
    __shared__ double red[kDotThreads / 32];
    double s = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += (double)x[i] * (double)y[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kDotThreads / 32; w++) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// out = sum of partial[0..n) in a fixed order (deterministic)
__global__ void dot_final(const double* __restrict__ partial, int n, double* __restrict__ out)
{
    __shared__ double red[kDotThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// phase 0: alpha = gamma / delta.  phase 1: beta = gammaNew / gamma, gamma = gammaNew,
// record ||r|| and sqrt(gamma) at slot it, it++.  phase 2: record slot 0.
__global__ void cg_scalars(double* sc, double* rnorm, double* gnorm, int phase)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (phase == 0) {
        const double d = sc[kDelta];
        sc[kAlpha] = d > 0.0 ? sc[kGamma] / d : 0.0;
    } else if (phase == 1) {
        const double g = sc[kGamma];
        sc[kBeta] = g > 0.0 ? sc[kGammaNew] / g : 0.0;
        sc[kGamma] = sc[kGammaNew];
        const int it = (int)sc[kIter] + 1;
        sc[kIter] = (double)it;
        rnorm[it] = sqrt(sc[kRr]);
        gnorm[it] = sqrt(sc[kGamma]);
    } else {
        sc[kIter] = 0.0;
        rnorm[0] = sqrt(sc[kRr]);
        gnorm[0] = sqrt(sc[kGamma]);
    }
}

// y += sign * alpha * x
__global__ void axpy(float* __restrict__ y, const float* __restrict__ x, const double* __restrict__ alpha,
                     float sign, size_t n)
{
    const float a = sign * (float)*alpha;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = fmaf(a, x[i], y[i]);
}

// p = s + beta * p
__global__ void xpby(float* __restrict__ p, const float* __restrict__ s, const double* __restrict__ beta, size_t n)
{
    const float b = (float)*beta;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = fmaf(b, p[i], s[i]);
}

// out[k][j] = in[k][j] sqrt(j dt) for 0 < j < nt, zero elsewhere: the prefolded
// weight's fold, the same factor ktmPrepareTraces and the demigration apply
__global__ void fold_samples(float* __restrict__ out, const float* __restrict__ in, int pitch, int nt,
                             float dt, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(i % (size_t)pitch);
        out[i] = (j > 0 && j < nt) ? in[i] * sqrtf((float)j * dt) : 0.0f;
    }
}

// r = d - q
__global__ void sub_into(float* __restrict__ r, const float* __restrict__ d, const float* __restrict__ q, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        r[i] = d[i] - q[i];
}

__global__ void fill(float* __restrict__ x, float v, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = v;
}

struct Lsm {
    Geometry g;
    const ktm_job* job;
    int pitch;
    size_t nd, nm;              // data and model lengths
    float *r, *q, *s, *p, *ones;
    float* rw;                  // prefolded weight: the folded residual the migration reads
    void* scratch; size_t scratchBytes; int slices;
    double *partial, *sc, *rnorm, *gnorm;
    cudaStream_t st;

    int dot(const float* x, const float* y, size_t n, double* out)
    {
        dot_partial<<<kDotBlocks, kDotThreads, 0, st>>>(x, y, n, partial);
        dot_final<<<1, kDotThreads, 0, st>>>(partial, kDotBlocks, out);
        KTM_CUDA_TRY(cudaGetLastError());
        return KTM_OK;
    }
    // data (packed F32) -> image; the prefolded weight folds the data first
    int migrate(const float* data, float* image)
    {
        const bool fold = job->weightMethod == KTM_WEIGHT_PREFOLD;
        if (fold) {
            fold_samples<<<blocks(nd), 256, 0, st>>>(rw, data, pitch, g.nt, g.dt, nd);
            KTM_CUDA_TRY(cudaGetLastError());
            data = rw;
        }
        FastArgs a;
        std::memset(&a, 0, sizeof(a));
        a.g = g;
        a.g.stride = pitch;
        a.midX = job->midX; a.midY = job->midY; a.offX = job->offX; a.offY = job->offY;
        a.traces = data; a.scale = ones; a.fmt = KTM_FMT_F32; a.pitch = pitch;
        a.weightMode = fold ? 2 : 0; a.weightMethod = job->weightMethod;
        a.vel = job->velocity; a.velCube = job->velocityCube;
        a.image = image; a.accumulate = 0;
        a.pick = job->pick; a.aperture = job->aperture; a.tileRun = job->tileRun;
        a.slices = slices; a.scratch = scratch; a.scratchBytes = scratchBytes;
        return launch_fast(a, st);
    }
    // image -> data (packed F32)
    int demigrate(const float* image, float* data)
    {
        return launch_demigrate(g, job->midX, job->midY, job->offX, job->offY, job->velocity,
                                job->velocityCube, image, data, pitch, job->pick, job->weightMethod,
                                job->aperture, 0, st);
    }
    unsigned blocks(size_t n) const
    {
        const size_t b = (n + 255) / 256;
        return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
    }
    int iteration(float* m)
    {
        int rc;
        if ((rc = demigrate(p, q))) return rc;                           // q = L p
        if ((rc = dot(q, q, nd, sc + kDelta))) return rc;                // delta = <q, q>
        cg_scalars<<<1, 32, 0, st>>>(sc, rnorm, gnorm, 0);               // alpha
        axpy<<<blocks(nm), 256, 0, st>>>(m, p, sc + kAlpha, 1.0f, nm);   // m += alpha p
        axpy<<<blocks(nd), 256, 0, st>>>(r, q, sc + kAlpha, -1.0f, nd);  // r -= alpha q
        if ((rc = migrate(r, s))) return rc;                             // s = L^T r
        if ((rc = dot(s, s, nm, sc + kGammaNew))) return rc;
        if ((rc = dot(r, r, nd, sc + kRr))) return rc;
        cg_scalars<<<1, 32, 0, st>>>(sc, rnorm, gnorm, 1);               // beta, gamma, norms
        xpby<<<blocks(nm), 256, 0, st>>>(p, s, sc + kBeta, nm);          // p = s + beta p
        KTM_CUDA_TRY(cudaGetLastError());
        return KTM_OK;
    }
};

}  // namespace
}  // namespace ktm

extern "C" int ktmLeastSquaresMigrate(const ktm_lsm* L)
{
    using namespace ktm;
    if (!L) return set_error(KTM_ERR_ARG, "NULL lsm");
    const ktm_job* j = &L->job;
    if (!j->deviceMemory) return set_error(KTM_ERR_ARG, "ktmLeastSquaresMigrate takes device memory");
    if (L->iterations < 0) return set_error(KTM_ERR_ARG, "negative iterations");
    if (j->pick != KTM_PICK_TRUNCATE && j->pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "bad pick %d", j->pick);
    if (j->weightMethod != KTM_WEIGHT_TABLE && j->weightMethod != KTM_WEIGHT_SQRT &&
        j->weightMethod != KTM_WEIGHT_PREFOLD)
        return set_error(KTM_ERR_ARG, "bad weightMethod %d", j->weightMethod);
    if (j->weightMethod == KTM_WEIGHT_PREFOLD && j->pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "the prefolded weight takes the linear pick");
    Lsm s;
    std::memset(&s, 0, sizeof(s));
    int rc = job_geometry(j, &s.g);
    if (rc) return rc;
    s.job = j;
    s.pitch = L->dataPitch;
    if (s.pitch < s.g.nt + 2 || s.pitch % 4 != 0)
        return set_error(KTM_ERR_ARG, "dataPitch must be >= tracePts + 2 and a multiple of 4");
    s.nd = (size_t)s.g.ntr * s.pitch;
    s.nm = (size_t)s.g.nx * s.g.ny * s.g.nz;
    if (!L->data || !L->model || !j->velocity || !j->midX || !j->midY || !j->offX || !j->offY)
        return set_error(KTM_ERR_ARG, "NULL pointer in the LSM job");
    if (s.nd == 0 || s.nm == 0) return set_error(KTM_ERR_ARG, "empty data or model");

    bool ownStream = false;
    s.st = static_cast<cudaStream_t>(j->stream);
    if (L->useGraph && s.st == nullptr) {
        // a capturable stream, ordered after the caller's work on the legacy stream
        // (which may have produced the data and the starting model)
        KTM_CUDA_TRY(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
        ownStream = true;
        cudaEvent_t ev;
        KTM_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, 0);
        cudaStreamWaitEvent(s.st, ev, 0);
        cudaEventDestroy(ev);
    }
    // workspace (all allocated before any capture)
    const int its = L->iterations;
    s.slices = (int)std::min<size_t>(64, std::max<size_t>(1, (size_t(256) << 20) / (s.nm * 4)));
    s.scratchBytes = (size_t)s.slices * s.nm * sizeof(float);
    const bool fold = j->weightMethod == KTM_WEIGHT_PREFOLD;
    // every piece starts on a 256-byte boundary (take() below)
    auto r256 = [](size_t n) { return (n + 255) / 256 * 256; };
    const size_t bytes = r256(kDotBlocks * sizeof(double)) + r256(kNScalars * sizeof(double)) +
                         2 * r256((its + 1) * sizeof(double)) + (fold ? 3 : 2) * r256(s.nd * 4) +
                         2 * r256(s.nm * 4) + r256((size_t)s.g.ntr * 4) + r256(s.scratchBytes);
    unsigned char* ws = nullptr;
    cudaError_t e = pool_malloc(reinterpret_cast<void**>(&ws), bytes, s.st);
    if (e != cudaSuccess) {
        if (ownStream) cudaStreamDestroy(s.st);
        return set_error(KTM_ERR_NOMEM, "ktmLeastSquaresMigrate: workspace of %zu bytes: %s", bytes,
                         cudaGetErrorString(e));
    }
    size_t off = 0;
    auto take = [&](size_t n) { unsigned char* p = ws + off; off += r256(n); return p; };
    s.partial = reinterpret_cast<double*>(take(kDotBlocks * sizeof(double)));
    s.sc = reinterpret_cast<double*>(take(kNScalars * sizeof(double)));
    s.rnorm = reinterpret_cast<double*>(take((its + 1) * sizeof(double)));
    s.gnorm = reinterpret_cast<double*>(take((its + 1) * sizeof(double)));
    s.r = reinterpret_cast<float*>(take(s.nd * 4));
    s.q = reinterpret_cast<float*>(take(s.nd * 4));
    s.s = reinterpret_cast<float*>(take(s.nm * 4));
    s.p = reinterpret_cast<float*>(take(s.nm * 4));
    s.ones = reinterpret_cast<float*>(take((size_t)s.g.ntr * 4));
    s.rw = fold ? reinterpret_cast<float*>(take(s.nd * 4)) : nullptr;
    s.scratch = take(s.scratchBytes);

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    do {
        fill<<<s.blocks(s.g.ntr), 256, 0, s.st>>>(s.ones, 1.0f, (size_t)s.g.ntr);
        // r = d - L m0, s = L^T r, p = s, gamma = <s, s>
        if ((rc = s.demigrate(L->model, s.q))) break;
        sub_into<<<s.blocks(s.nd), 256, 0, s.st>>>(s.r, L->data, s.q, s.nd);
        if ((rc = s.migrate(s.r, s.s))) break;
        e = cudaMemcpyAsync(s.p, s.s, s.nm * 4, cudaMemcpyDeviceToDevice, s.st);
        if (e != cudaSuccess) { rc = set_error(KTM_ERR_CUDA, "copy: %s", cudaGetErrorString(e)); break; }
        if ((rc = s.dot(s.s, s.s, s.nm, s.sc + kGamma))) break;
        if ((rc = s.dot(s.r, s.r, s.nd, s.sc + kRr))) break;
        cg_scalars<<<1, 32, 0, s.st>>>(s.sc, s.rnorm, s.gnorm, 2);
        if (its == 0) break;
        if (L->useGraph) {
            e = cudaStreamBeginCapture(s.st, cudaStreamCaptureModeRelaxed);
            if (e != cudaSuccess) { rc = set_error(KTM_ERR_CUDA, "capture: %s", cudaGetErrorString(e)); break; }
            rc = s.iteration(L->model);
            e = cudaStreamEndCapture(s.st, &graph);
            if (rc) break;
            if (e != cudaSuccess) { rc = set_error(KTM_ERR_CUDA, "end capture: %s", cudaGetErrorString(e)); break; }
            e = cudaGraphInstantiate(&exec, graph, 0);
            if (e != cudaSuccess) { rc = set_error(KTM_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e)); break; }
            for (int i = 0; i < its && e == cudaSuccess; i++) e = cudaGraphLaunch(exec, s.st);
            if (e != cudaSuccess) { rc = set_error(KTM_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e)); break; }
        } else {
            for (int i = 0; i < its && !rc; i++) rc = s.iteration(L->model);
        }
    } while (false);
    if (!rc && (L->residualNorms || L->gradientNorms)) {
        if (L->residualNorms)
            e = cudaMemcpyAsync(L->residualNorms, s.rnorm, (its + 1) * sizeof(double), cudaMemcpyDeviceToHost, s.st);
        if (e == cudaSuccess && L->gradientNorms)
            e = cudaMemcpyAsync(L->gradientNorms, s.gnorm, (its + 1) * sizeof(double), cudaMemcpyDeviceToHost, s.st);
        if (e != cudaSuccess) rc = set_error(KTM_ERR_CUDA, "norms: %s", cudaGetErrorString(e));
    }
    cudaError_t se = cudaStreamSynchronize(s.st);
    if (!rc && se != cudaSuccess) rc = set_error(KTM_ERR_CUDA, "lsm: %s", cudaGetErrorString(se));
    unsigned stalls = 0;
    if (!rc) rc = take_wait_stalls(s.st, false, &stalls);
    if (!rc && stalls) rc = set_error(KTM_ERR_TIMEOUT, "lsm: %u bounded device wait(s) ran out", stalls);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFreeAsync(ws, s.st);
    cudaStreamSynchronize(s.st);
    if (ownStream) cudaStreamDestroy(s.st);
    return rc ? rc : set_ok();
}
