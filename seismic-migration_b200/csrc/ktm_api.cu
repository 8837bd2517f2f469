// ktm_api.cu -- the C ABI of libktm.so: status, the drop-in entry points that
// replace ktmMigrationCPU / ktmMigrationGPU, and the extended job API.
#include "ktm_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

namespace ktm {

namespace {
thread_local int tl_code = KTM_OK;
thread_local char tl_msg[512] = "";
}  // namespace

int set_error(int code, const char* fmt, ...)
{
    tl_code = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(tl_msg, sizeof(tl_msg), fmt, ap);
    va_end(ap);
    return code;
}

int set_ok()
{
    tl_code = KTM_OK;
    tl_msg[0] = 0;
    return KTM_OK;
}

namespace {
constexpr int kPoolDevices = 64;
std::mutex g_poolMu;
cudaMemPool_t g_pool[kPoolDevices];
bool g_poolTried[kPoolDevices];
std::atomic<unsigned long long> g_poolCalls{0};   // pool_malloc calls since the library loaded
}  // namespace

cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t s)
{
    g_poolCalls.fetch_add(1, std::memory_order_relaxed);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = nullptr;
    if (dev >= 0 && dev < kPoolDevices) {
        std::lock_guard<std::mutex> lk(g_poolMu);
        if (!g_poolTried[dev]) {
            g_poolTried[dev] = true;
            cudaMemPoolProps props;
            std::memset(&props, 0, sizeof(props));
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t created = nullptr;
            if (cudaMemPoolCreate(&created, &props) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
                g_pool[dev] = created;
            } else {
                cudaGetLastError();
            }
        }
        pool = g_pool[dev];
    }
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaMallocAsync(p, bytes, s);
}

namespace {

bool grid_ok(const imageGrid& g) { return g.imagePnts >= 0; }

int make_geometry(const ktm_job* j, Geometry* g)
{
    if (!grid_ok(j->imageX) || !grid_ok(j->imageY) || !grid_ok(j->imageZ))
        return set_error(KTM_ERR_ARG, "image axis with negative point count");
    if (j->config.traceNo < 0 || j->config.tracePts < 0)
        return set_error(KTM_ERR_ARG, "negative traceNo or tracePts");
    if (!(j->config.traceSampleRate > 0.0f))
        return set_error(KTM_ERR_ARG, "traceSampleRate must be > 0");
    const long long cols = (long long)j->imageX.imagePnts * j->imageY.imagePnts;
    if (cols > 0x7fffffffLL || cols * j->imageZ.imagePnts > (1LL << 40))
        return set_error(KTM_ERR_LIMIT, "image too large");
    g->nx = j->imageX.imagePnts; g->ny = j->imageY.imagePnts; g->nz = j->imageZ.imagePnts;
    g->x0 = j->imageX.imageStart; g->dx = j->imageX.imageStep;
    g->y0 = j->imageY.imageStart; g->dy = j->imageY.imageStep;
    g->z0 = j->imageZ.imageStart; g->dz = j->imageZ.imageStep;
    g->ntr = j->config.traceNo; g->nt = j->config.tracePts;
    g->stride = j->traceStride > 0 ? j->traceStride : j->config.tracePts;
    if (g->stride < g->nt) return set_error(KTM_ERR_ARG, "traceStride < tracePts");
    g->dt = j->config.traceSampleRate;
    return KTM_OK;
}

size_t fmt_bytes(int fmt) { return (fmt == KTM_FMT_F32 || fmt == KTM_FMT_IBM32) ? 4 : 2; }

// Device copies of a host-memory job (freed in the destructor, stream-ordered).
struct Staged {
    cudaStream_t s;
    std::vector<void*> ptrs;
    explicit Staged(cudaStream_t st) : s(st) {}
    ~Staged()
    {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
    int alloc(void** p, size_t bytes)
    {
        *p = nullptr;
        if (bytes == 0) return KTM_OK;
        KTM_CUDA_TRY(pool_malloc(p, bytes, s));
        ptrs.push_back(*p);
        return KTM_OK;
    }
    template <class T>
    int upload(const T* host, size_t bytes, const T** dev)
    {
        *dev = nullptr;
        if (!host || bytes == 0) return KTM_OK;
        void* d;
        int rc = alloc(&d, bytes);
        if (rc) return rc;
        KTM_CUDA_TRY(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, s));
        *dev = static_cast<const T*>(d);
        return KTM_OK;
    }
};

int run_device(const ktm_job* j, const Geometry& g, const float* midX, const float* midY,
               const float* offX, const float* offY, const void* traces, const float* scale,
               const float* vel, float* image, cudaStream_t s)
{
    if (j->mode == KTM_MODE_REFERENCE) {
        const bool ibm = j->traceFormat == KTM_FMT_IBM32;
        if ((j->traceFormat != KTM_FMT_F32 && !ibm) || j->pick != KTM_PICK_TRUNCATE ||
            j->velocityCube || j->aperture > 0.0f || j->tracesPrefolded || scale)
            return set_error(KTM_ERR_ARG,
                             "reference mode takes F32 or IBM-32 traces, truncating pick, no "
                             "aperture, no scale and a 1-D velocity (psktmCPU.c semantics)");
        if (!ibm)
            return launch_reference(g, midX, midY, offX, offY, static_cast<const float*>(traces),
                                    vel, image, j->accumulate, j->tileRun, s);
        // IBM words: convert on the device (ioFunctions.c:4-40), then migrate
        const size_t n = (size_t)g.ntr * g.stride;
        void* conv = nullptr;
        if (n) KTM_CUDA_TRY(pool_malloc(&conv, n * 4, s));
        int rc = ibm_to_ieee(static_cast<const uint32_t*>(traces), static_cast<float*>(conv), n, s);
        if (!rc)
            rc = launch_reference(g, midX, midY, offX, offY, static_cast<const float*>(conv), vel,
                                  image, j->accumulate, j->tileRun, s);
        if (conv) cudaFreeAsync(conv, s);
        return rc;
    }
    if (j->mode == KTM_MODE_FAST) {
        FastArgs a;
        std::memset(&a, 0, sizeof(a));
        a.g = g; a.midX = midX; a.midY = midY; a.offX = offX; a.offY = offY;
        a.vel = vel; a.velCube = j->velocityCube;
        a.image = image; a.accumulate = j->accumulate;
        a.pick = j->pick; a.aperture = j->aperture;
        a.tileRun = j->tileRun; a.tileCols = j->tileCols; a.chunkCap = j->tileChunk;
        a.pairsEvaluated = j->pairsEvaluated;
        // weight sqrt(t): from the kernel's table / sqrt (0) or folded into the packed samples (2)
        a.weightMode = (j->tracesPacked && j->tracesPrefolded) ? 2 : 0;
        if (j->weightMethod != KTM_WEIGHT_TABLE && j->weightMethod != KTM_WEIGHT_SQRT &&
            j->weightMethod != KTM_WEIGHT_PREFOLD)
            return set_error(KTM_ERR_ARG, "bad weightMethod %d", j->weightMethod);
        const int wantPrefold = j->weightMethod == KTM_WEIGHT_PREFOLD;
        if (wantPrefold && j->pick != KTM_PICK_LINEAR)
            return set_error(KTM_ERR_ARG, "KTM_WEIGHT_PREFOLD takes the linear pick");
        if (wantPrefold && j->tracesPacked && !j->tracesPrefolded)
            return set_error(KTM_ERR_ARG, "KTM_WEIGHT_PREFOLD with packed traces: prepare them "
                                          "with prefold = 1");
        a.weightMethod = wantPrefold ? KTM_WEIGHT_TABLE : j->weightMethod;
        if (j->tracesPacked) {
            if (j->traceFormat == KTM_FMT_IBM32)
                return set_error(KTM_ERR_ARG, "packed traces cannot be IBM-32");
            a.traces = traces; a.scale = scale; a.fmt = j->traceFormat; a.pitch = g.stride;
            if (!scale) return set_error(KTM_ERR_ARG, "packed traces need traceScale");
            return launch_fast(a, s);
        }
        // raw traces: filter and pack into a temporary set (job->rho, job->packFormat)
        if (j->packFormat < KTM_FMT_F32 || j->packFormat > KTM_FMT_BF16)
            return set_error(KTM_ERR_ARG, "bad packFormat %d", j->packFormat);
        const float* in = static_cast<const float*>(traces);
        void* packed = nullptr;
        float* pscale = nullptr;
        const float* src32 = in;
        void* widened = nullptr;
        int rc = KTM_OK;
        if (j->traceFormat == KTM_FMT_F16 || j->traceFormat == KTM_FMT_BF16) {
            // half-precision input: widen (times its scale) to F32 first
            rc = widen_traces(traces, j->traceFormat, scale, g.ntr, g.nt, g.stride, &widened, s);
            if (rc) return rc;
            src32 = static_cast<const float*>(widened);
        }
        const int pitch = packed_pitch(g.nt, j->packFormat);
        const size_t esize = j->packFormat == KTM_FMT_F32 ? 4 : 2;
        cudaError_t e = pool_malloc(&packed, (size_t)g.ntr * pitch * esize, s);
        if (e == cudaSuccess) e = pool_malloc(reinterpret_cast<void**>(&pscale), (size_t)g.ntr * 4, s);
        if (e != cudaSuccess) {
            rc = set_error(KTM_ERR_NOMEM, "fast path: packing buffer: %s", cudaGetErrorString(e));
        } else {
            ktm_prep p;
            std::memset(&p, 0, sizeof(p));
            p.traceNo = g.ntr; p.tracePts = g.nt;
            p.inStride = widened ? g.nt : g.stride;
            p.sampleRate = g.dt; p.in = src32; p.prefold = wantPrefold; p.rho = j->rho;
            // IBM words are converted inside the preparation pass
            p.inFormat = j->traceFormat == KTM_FMT_IBM32 ? KTM_FMT_IBM32 : KTM_FMT_F32;
            p.outFormat = j->packFormat; p.outPitch = pitch; p.out = packed; p.outScale = pscale;
            p.stream = s;
            rc = prepare_traces(&p);
            if (!rc) {
                a.traces = packed; a.scale = pscale; a.fmt = j->packFormat; a.pitch = pitch;
                a.weightMode = wantPrefold ? 2 : 0;
                rc = launch_fast(a, s);
            }
        }
        if (packed) cudaFreeAsync(packed, s);
        if (pscale) cudaFreeAsync(pscale, s);
        if (widened) cudaFreeAsync(widened, s);
        return rc;
    }
    return set_error(KTM_ERR_ARG, "ktmMigrate: mode must be REFERENCE or FAST "
                                  "(FP64 output goes through ktmMigrateColumnsF64)");
}

// KTM_ERR_TIMEOUT when a bounded device wait ran out since the last check
int check_waits(cudaStream_t s, bool deviceSync)
{
    unsigned n = 0;
    const int rc = take_wait_stalls(s, deviceSync, &n);
    if (rc) return rc;
    if (n) return set_error(KTM_ERR_TIMEOUT, "%u bounded device wait(s) for a bulk trace copy ran out", n);
    return set_ok();
}

// allowF64: KTM_FMT_F64 traces (the FP64 device evaluation only)
int check_job(const ktm_job* j, bool allowF64 = false)
{
    if (!j) return set_error(KTM_ERR_ARG, "NULL job");
    if (j->traceFormat == KTM_FMT_F64 && !allowF64)
        return set_error(KTM_ERR_ARG, "KTM_FMT_F64 traces are taken by ktmMigrateColumnsF64 only");
    if (j->traceFormat < KTM_FMT_F32 || j->traceFormat > KTM_FMT_F64)
        return set_error(KTM_ERR_ARG, "bad traceFormat %d", j->traceFormat);
    if (j->traceFormat == KTM_FMT_IBM32 && (j->traceScale || j->tracesPacked))
        return set_error(KTM_ERR_ARG, "IBM-32 traces are raw: no traceScale, not packed");
    if (j->pick != KTM_PICK_TRUNCATE && j->pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "bad pick %d", j->pick);
    const bool needTraces = j->config.traceNo > 0;
    if (needTraces && (!j->midX || !j->midY || !j->offX || !j->offY || !j->traces))
        return set_error(KTM_ERR_ARG, "NULL coordinate or trace pointer");
    if (!j->velocity && (long long)j->imageZ.imagePnts > 0)
        return set_error(KTM_ERR_ARG, "NULL velocity");
    if (!j->image && (long long)j->imageX.imagePnts * j->imageY.imagePnts * j->imageZ.imagePnts > 0)
        return set_error(KTM_ERR_ARG, "NULL image");
    return KTM_OK;
}

int migrate_impl(const ktm_job* j)
{
    int rc = check_job(j);
    if (rc) return rc;
    Geometry g;
    rc = make_geometry(j, &g);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(j->stream);
    if (j->deviceMemory) {
        rc = run_device(j, g, j->midX, j->midY, j->offX, j->offY, j->traces, j->traceScale,
                        j->velocity, j->image, s);
        return rc ? rc : set_ok();
    }
    // host buffers: copy in, run, copy out, synchronise
    const size_t ntr = (size_t)g.ntr, nimg = (size_t)g.nx * g.ny * g.nz;
    const size_t nvel = j->velocityCube ? nimg : (size_t)g.nz;
    const float *dmx, *dmy, *dox, *doy, *dsc, *dvel;
    const unsigned char* dtr;
    void* dimg = nullptr;
    {
        Staged st(s);
        if ((rc = st.upload(j->midX, ntr * 4, &dmx)) || (rc = st.upload(j->midY, ntr * 4, &dmy)) ||
            (rc = st.upload(j->offX, ntr * 4, &dox)) || (rc = st.upload(j->offY, ntr * 4, &doy)) ||
            (rc = st.upload(static_cast<const unsigned char*>(j->traces),
                            ntr * g.stride * fmt_bytes(j->traceFormat), &dtr)) ||
            (rc = st.upload(j->traceScale, j->traceScale ? ntr * 4 : 0, &dsc)) ||
            (rc = st.upload(j->velocity, nvel * 4, &dvel)) || (rc = st.alloc(&dimg, nimg * 4)))
            return rc;
        if (j->accumulate && nimg)
            KTM_CUDA_TRY(cudaMemcpyAsync(dimg, j->image, nimg * 4, cudaMemcpyHostToDevice, s));
        rc = run_device(j, g, dmx, dmy, dox, doy, dtr, dsc, dvel, static_cast<float*>(dimg), s);
        if (rc) return rc;
        if (nimg)
            KTM_CUDA_TRY(cudaMemcpyAsync(j->image, dimg, nimg * 4, cudaMemcpyDeviceToHost, s));
    }
    KTM_CUDA_TRY(cudaStreamSynchronize(s));
    return check_waits(s, false);
}

void dropin(imageGrid* imageX, imageGrid* imageY, imageGrid* imageZ, jobParams* config,
            float* midX, float* midY, float* offX, float* offY, float* traces, float* slowness,
            float* image)
{
    if (!imageX || !imageY || !imageZ || !config) {
        set_error(KTM_ERR_ARG, "NULL grid or config");
        return;
    }
    ktm_job j;
    ktmJobInit(&j);
    j.imageX = *imageX; j.imageY = *imageY; j.imageZ = *imageZ; j.config = *config;
    j.midX = midX; j.midY = midY; j.offX = offX; j.offY = offY;
    j.traces = traces; j.velocity = slowness; j.image = image;
    j.mode = KTM_MODE_REFERENCE;
    j.pick = KTM_PICK_TRUNCATE;
    j.deviceMemory = 0;
    migrate_impl(&j);
}

}  // namespace
}  // namespace ktm

extern "C" {

int ktmCheckDeviceWaits(void)
{
    return ktm::check_waits(0, true);
}

int ktmSelfTestDeviceWait(int stall, int limitMs)
{
    if (limitMs <= 0 || limitMs > 10000) return ktm::set_error(KTM_ERR_ARG, "limitMs must be in 1..10000");
    unsigned sum = 0;
    int rc = ktm::wait_selftest(stall ? 1 : 0, (unsigned long long)limitMs * 1000000ull, &sum);
    if (rc) return rc;
    rc = ktm::check_waits(0, false);
    if (rc) return rc;
    if (sum != 16384u * 0x01010101u) return ktm::set_error(KTM_ERR_CUDA, "bulk copy landed wrong bytes");
    return ktm::set_ok();
}

int ktmReleaseMemory(void)
{
    std::lock_guard<std::mutex> lk(ktm::g_poolMu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < ktm::kPoolDevices; d++) {
        if (!ktm::g_pool[d]) continue;
        cudaError_t e = cudaSetDevice(d);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemPoolTrimTo(ktm::g_pool[d], 0);
        if (e != cudaSuccess) {
            cudaSetDevice(cur);
            return ktm::set_error(KTM_ERR_CUDA, "ktmReleaseMemory: %s", cudaGetErrorString(e));
        }
    }
    cudaSetDevice(cur);
    return ktm::set_ok();
}

int ktmMemoryStats(unsigned long long* allocations, size_t* reservedBytes, size_t* usedBytes)
{
    if (allocations) *allocations = ktm::g_poolCalls.load(std::memory_order_relaxed);
    int dev = 0;
    if (reservedBytes) *reservedBytes = 0;
    if (usedBytes) *usedBytes = 0;
    if (!reservedBytes && !usedBytes) return ktm::set_ok();
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ktm::set_error(KTM_ERR_CUDA, "ktmMemoryStats: %s", cudaGetErrorString(e));
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(ktm::g_poolMu);
        if (dev >= 0 && dev < ktm::kPoolDevices) pool = ktm::g_pool[dev];
    }
    if (!pool) return ktm::set_ok();                 // nothing allocated on this device yet
    uint64_t v = 0;
    if (reservedBytes) {
        e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v);
        if (e != cudaSuccess) return ktm::set_error(KTM_ERR_CUDA, "ktmMemoryStats: %s", cudaGetErrorString(e));
        *reservedBytes = (size_t)v;
    }
    if (usedBytes) {
        e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &v);
        if (e != cudaSuccess) return ktm::set_error(KTM_ERR_CUDA, "ktmMemoryStats: %s", cudaGetErrorString(e));
        *usedBytes = (size_t)v;
    }
    return ktm::set_ok();
}

// status hooks of the host-side file I/O (ktm_io.c)
int ktm_io_error(int code, const char* msg) { return ktm::set_error(code, "%s", msg); }
int ktm_io_ok(void) { return ktm::set_ok(); }

int ktmGetLastError(void) { return ktm::tl_code; }
const char* ktmGetLastErrorMessage(void) { return ktm::tl_msg; }

const char* ktmGetErrorString(int code)
{
    switch (code) {
        case KTM_OK: return "ok";
        case KTM_ERR_ARG: return "invalid argument";
        case KTM_ERR_CUDA: return "CUDA runtime error";
        case KTM_ERR_NOMEM: return "out of memory";
        case KTM_ERR_LIMIT: return "size beyond a kernel limit";
        case KTM_ERR_IO: return "file I/O error";
        case KTM_ERR_TIMEOUT: return "device wait timed out";
        case KTM_ERR_NODEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

void ktmJobInit(ktm_job* job)
{
    if (!job) return;
    std::memset(job, 0, sizeof(*job));
    job->mode = KTM_MODE_FAST;
    job->pick = KTM_PICK_LINEAR;
    job->traceFormat = KTM_FMT_F32;
}

int ktmMigrate(const ktm_job* job) { return ktm::migrate_impl(job); }

size_t ktmJobStructSize(void) { return sizeof(ktm_job); }

void ktmMigrationCPU(imageGrid* imageX, imageGrid* imageY, imageGrid* imageZ, jobParams* config,
                     float* midX, float* midY, float* offX, float* offY, float* traces,
                     float* slowness, float* image)
{
    ktm::dropin(imageX, imageY, imageZ, config, midX, midY, offX, offY, traces, slowness, image);
}

void ktmMigrationGPU(imageGrid* imageX, imageGrid* imageY, imageGrid* imageZ, jobParams* config,
                     float* midX, float* midY, float* offX, float* offY, float* traces,
                     float* slowness, float* image)
{
    ktm::dropin(imageX, imageY, imageZ, config, midX, midY, offX, offY, traces, slowness, image);
}

void initThreeAxes(imageGrid* imageX, imageGrid* imageY, imageGrid* imageZ, float* imageXX,
                   float* imageYY, float* imageZZ)
{
    // psktmFunctions.c:26-33 (host code built with -ffp-contract=off: the product
    // and the sum are rounded separately, as in the reference build)
    for (int i = 0; i < imageX->imagePnts; i++) {
        float p = (float)i * imageX->imageStep;
        imageXX[i] = imageX->imageStart + p;
    }
    initTwoAxes(imageY, imageZ, imageYY, imageZZ);
}

void initTwoAxes(imageGrid* imageY, imageGrid* imageZ, float* imageYY, float* imageZZ)
{
    // psktmFunctions.c:9-13
    for (int i = 0; i < imageY->imagePnts; i++) {
        float p = (float)i * imageY->imageStep;
        imageYY[i] = imageY->imageStart + p;
    }
    for (int i = 0; i < imageZ->imagePnts; i++) {
        float p = (float)i * imageZ->imageStep;
        imageZZ[i] = imageZ->imageStart + p;
    }
}

int ktmMigrateColumnsF64(const ktm_job* job, const int* columns, int ncols, double* out)
{
    int rc = ktm::check_job(job, true);
    if (rc) return rc;
    if (!job->deviceMemory)
        return ktm::set_error(KTM_ERR_ARG, "ktmMigrateColumnsF64 takes device memory");
    if (job->traceFormat == KTM_FMT_F64 && (job->tracesPacked || job->traceScale))
        return ktm::set_error(KTM_ERR_ARG, "ktmMigrateColumnsF64: F64 traces are raw (not packed, "
                                           "no traceScale)");
    if (ncols < 0 || (!out && ncols > 0)) return ktm::set_error(KTM_ERR_ARG, "bad column list");
    if (job->traceFormat == KTM_FMT_IBM32)
        return ktm::set_error(KTM_ERR_ARG, "ktmMigrateColumnsF64: convert IBM-32 traces first "
                                           "(ktmIBM32toIEEEDevice)");
    ktm::Geometry g;
    rc = ktm::make_geometry(job, &g);
    if (rc) return rc;
    ktm::FastArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = g; a.midX = job->midX; a.midY = job->midY; a.offX = job->offX; a.offY = job->offY;
    a.traces = job->traces; a.scale = job->traceScale; a.fmt = job->traceFormat; a.pitch = g.stride;
    a.weightMode = job->tracesPrefolded ? 2 : 0;
    a.vel = job->velocity; a.velCube = job->velocityCube;
    a.pick = job->pick; a.aperture = job->aperture;
    rc = ktm::launch_f64_columns(a, columns, ncols, out, static_cast<cudaStream_t>(job->stream));
    return rc ? rc : ktm::set_ok();
}

}  // extern "C"

namespace ktm {
int job_geometry(const ktm_job* j, Geometry* g) { return make_geometry(j, g); }
}  // namespace ktm

extern "C" int ktmDemigrate(const ktm_job* job, float* data, int dataPitch)
{
    using namespace ktm;
    if (!job) return set_error(KTM_ERR_ARG, "NULL job");
    if (!job->deviceMemory) return set_error(KTM_ERR_ARG, "ktmDemigrate takes device memory");
    if (job->pick != KTM_PICK_TRUNCATE && job->pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "bad pick %d", job->pick);
    if (job->weightMethod != KTM_WEIGHT_TABLE && job->weightMethod != KTM_WEIGHT_SQRT &&
        job->weightMethod != KTM_WEIGHT_PREFOLD)
        return set_error(KTM_ERR_ARG, "bad weightMethod %d", job->weightMethod);
    if (job->weightMethod == KTM_WEIGHT_PREFOLD && job->pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "the prefolded weight takes the linear pick");
    Geometry g;
    int rc = make_geometry(job, &g);
    if (rc) return rc;
    const long long nimg = (long long)g.nx * g.ny * g.nz;
    if (g.ntr > 0 && (!job->midX || !job->midY || !job->offX || !job->offY || !data))
        return set_error(KTM_ERR_ARG, "NULL coordinate or data pointer");
    if (nimg > 0 && g.ntr > 0 && (!job->image || !job->velocity))
        return set_error(KTM_ERR_ARG, "NULL model or velocity");
    rc = launch_demigrate(g, job->midX, job->midY, job->offX, job->offY, job->velocity,
                          job->velocityCube, job->image, data, dataPitch, job->pick,
                          job->weightMethod, job->aperture, job->accumulate,
                          static_cast<cudaStream_t>(job->stream));
    return rc ? rc : set_ok();
}

extern "C" int ktmVrmsGradient(const ktm_job* job, float* grad)
{
    using namespace ktm;
    if (!job) return set_error(KTM_ERR_ARG, "NULL job");
    if (!job->deviceMemory || !job->tracesPacked)
        return set_error(KTM_ERR_ARG, "ktmVrmsGradient takes device memory and a packed trace set");
    int rc = check_job(job);
    if (rc) return rc;
    Geometry g;
    rc = make_geometry(job, &g);
    if (rc) return rc;
    if (!grad && (long long)g.nx * g.ny * g.nz > 0) return set_error(KTM_ERR_ARG, "NULL grad");
    if (!job->traceScale) return set_error(KTM_ERR_ARG, "packed traces need traceScale");
    FastArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = g; a.midX = job->midX; a.midY = job->midY; a.offX = job->offX; a.offY = job->offY;
    a.traces = job->traces; a.scale = job->traceScale; a.fmt = job->traceFormat; a.pitch = g.stride;
    a.weightMode = job->tracesPrefolded ? 2 : 0;
    a.weightMethod = job->weightMethod;
    a.vel = job->velocity; a.velCube = job->velocityCube;
    a.image = grad; a.accumulate = 0;
    a.pick = job->pick; a.aperture = job->aperture;
    a.tileRun = job->tileRun;
    a.grad = 1;
    rc = launch_fast(a, static_cast<cudaStream_t>(job->stream));
    return rc ? rc : set_ok();
}

namespace ktm {

// FastArgs of a device-memory FAST job on a packed trace set.
int packed_args(const ktm_job* j, FastArgs* a)
{
    if (!j) return set_error(KTM_ERR_ARG, "NULL job");
    if (!j->deviceMemory || !j->tracesPacked || j->mode != KTM_MODE_FAST)
        return set_error(KTM_ERR_ARG, "batched and tuned launches take FAST mode, device memory "
                                      "and packed traces");
    int rc = check_job(j);
    if (rc) return rc;
    if (j->weightMethod != KTM_WEIGHT_TABLE && j->weightMethod != KTM_WEIGHT_SQRT &&
        !(j->weightMethod == KTM_WEIGHT_PREFOLD && j->tracesPrefolded))
        return set_error(KTM_ERR_ARG, "bad weightMethod %d", j->weightMethod);
    std::memset(a, 0, sizeof(*a));
    rc = make_geometry(j, &a->g);
    if (rc) return rc;
    if (!j->traceScale && j->config.traceNo > 0) return set_error(KTM_ERR_ARG, "packed traces need traceScale");
    a->midX = j->midX; a->midY = j->midY; a->offX = j->offX; a->offY = j->offY;
    a->traces = j->traces; a->scale = j->traceScale; a->fmt = j->traceFormat; a->pitch = a->g.stride;
    a->weightMode = j->tracesPrefolded ? 2 : 0;
    a->weightMethod = j->weightMethod == KTM_WEIGHT_PREFOLD ? KTM_WEIGHT_TABLE : j->weightMethod;
    a->vel = j->velocity; a->velCube = j->velocityCube;
    a->image = j->image; a->accumulate = j->accumulate;
    a->pick = j->pick; a->aperture = j->aperture;
    a->tileRun = j->tileRun;
    a->tileCols = j->tileCols;
    a->chunkCap = j->tileChunk;
    a->pairsEvaluated = j->pairsEvaluated;
    return KTM_OK;
}

namespace {

struct TuneKey {
    int nx, ny, nz, nt, fmt, pick, weightMode, weightMethod;
    bool operator<(const TuneKey& o) const
    {
        return std::memcmp(this, &o, sizeof(TuneKey)) < 0;
    }
};
std::mutex g_tuneMu;
std::map<TuneKey, ktm_tile> g_tuned;

// The fast kernel's CTA shapes: columns per CTA and CTAs resident per SM (ktm_fast.cu).
int ctas_per_sm(int cols) { return cols == 8 ? 3 : cols == 12 ? 2 : 1; }

// Candidate tiles of a job: tau runs 512 / 384 / 256 x CTA shapes (24 x 1, 12 x 2,
// 8 x 3 columns x CTAs per SM where the path is built for them, else 24 x 1) x
// traces per chunk (as many as fit, or at most 8).
std::vector<ktm_tile> tile_candidates(const FastArgs& a)
{
    const bool tunable = a.pick == KTM_PICK_LINEAR &&
                         (a.weightMode == 2 || a.weightMethod == KTM_WEIGHT_TABLE);
    std::vector<ktm_tile> out;
    for (int run : {512, 384, 256})
        for (int cols : {24, 12, 8}) {
            if (!tunable && cols != 24) continue;
            for (int chunk : {0, 8}) {
                ktm_tile t;
                std::memset(&t, 0, sizeof(t));
                t.tileRun = run; t.tileCols = cols; t.tileChunk = chunk;
                t.ctasPerSm = ctas_per_sm(cols);
                out.push_back(t);
            }
        }
    return out;
}

TuneKey tune_key(const FastArgs& a)
{
    TuneKey key;
    std::memset(&key, 0, sizeof(key));
    key.nx = a.g.nx; key.ny = a.g.ny; key.nz = a.g.nz; key.nt = a.g.nt; key.fmt = a.fmt;
    key.pick = a.pick; key.weightMode = a.weightMode; key.weightMethod = a.weightMethod;
    return key;
}

// Times every candidate on up to kTuneTraces of the job's traces (one warm-up and
// two timed launches each, CUDA events on the job's stream) and returns the fastest.
constexpr int kTuneTraces = 4096;
int autotune_tile(const ktm_job* job, ktm_tile* best)
{
    FastArgs a;
    int rc = packed_args(job, &a);
    if (rc) return rc;
    const TuneKey key = tune_key(a);
    {
        std::lock_guard<std::mutex> lock(g_tuneMu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            *best = it->second;
            return KTM_OK;
        }
    }
    if ((long long)a.g.nx * a.g.ny * a.g.nz == 0 || a.g.ntr == 0) {
        // nothing to time: the default shape
        std::memset(best, 0, sizeof(*best));
        best->tileRun = 32 * 16; best->tileCols = 24; best->ctasPerSm = 1;
        return KTM_OK;
    }
    cudaStream_t s = static_cast<cudaStream_t>(job->stream);
    a.g.ntr = std::min(a.g.ntr, kTuneTraces);
    a.accumulate = 0;
    a.pairsEvaluated = nullptr;
    cudaEvent_t e0, e1;
    KTM_CUDA_TRY(cudaEventCreate(&e0));
    KTM_CUDA_TRY(cudaEventCreate(&e1));
    ktm_tile chosen;
    std::memset(&chosen, 0, sizeof(chosen));
    float bestMs = 3.0e38f;
    for (ktm_tile t : tile_candidates(a)) {
        a.tileRun = t.tileRun; a.tileCols = t.tileCols; a.chunkCap = t.tileChunk;
        if ((rc = launch_fast(a, s))) break;               // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 2 && !rc; r++) rc = launch_fast(a, s);
        cudaEventRecord(e1, s);
        if (rc) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = set_error(KTM_ERR_CUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        t.ms = ms / 2.0f;
        if (t.ms < bestMs) { bestMs = t.ms; chosen = t; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lock(g_tuneMu);
        g_tuned[key] = chosen;
    }
    *best = chosen;
    return KTM_OK;
}

}  // namespace
}  // namespace ktm

extern "C" int ktmMigrateBatch(const ktm_job* jobs, int njobs, void* stream)
{
    using namespace ktm;
    if (njobs < 0 || (njobs > 0 && !jobs)) return set_error(KTM_ERR_ARG, "bad job list");
    std::vector<FastArgs> args(njobs);
    for (int j = 0; j < njobs; j++) {
        int rc = packed_args(&jobs[j], &args[j]);
        if (rc) return rc;
        if (!jobs[j].image && (long long)args[j].g.nx * args[j].g.ny * args[j].g.nz > 0)
            return set_error(KTM_ERR_ARG, "job %d: NULL image", j);
    }
    int rc = launch_batch(args.data(), njobs, static_cast<cudaStream_t>(stream));
    return rc ? rc : set_ok();
}

extern "C" int ktmAutotuneTile(const ktm_job* job, ktm_tile* best)
{
    using namespace ktm;
    if (!best) return set_error(KTM_ERR_ARG, "NULL tile");
    const int rc = autotune_tile(job, best);
    return rc ? rc : set_ok();
}

extern "C" int ktmAutotune(const ktm_job* job, int* tileRun)
{
    using namespace ktm;
    if (!tileRun) return set_error(KTM_ERR_ARG, "NULL tileRun");
    ktm_tile t;
    const int rc = autotune_tile(job, &t);
    if (rc) return rc;
    *tileRun = t.tileRun;
    return set_ok();
}

extern "C" int ktmTileCandidates(const ktm_job* job, ktm_tile* out, int capacity, int* count)
{
    using namespace ktm;
    if (!count || capacity < 0 || (capacity > 0 && !out)) return set_error(KTM_ERR_ARG, "bad output");
    FastArgs a;
    const int rc = packed_args(job, &a);
    if (rc) return rc;
    const std::vector<ktm_tile> c = tile_candidates(a);
    *count = (int)c.size();
    for (int i = 0; i < (int)c.size() && i < capacity; i++) out[i] = c[i];
    return set_ok();
}
