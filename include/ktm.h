/*
 * ktm.h -- C ABI of libktm.so, a B200 (sm_100a) prestack Kirchhoff time
 * migration (PSTM) library that is a drop-in for the psktmCPU.c /
 * psktmFunctions.c path of wjb19/seismic-migration.
 *
 * Conventions shared by every entry point
 *   - Image layout: float[Nx][Ny][Nz], tau fastest (psktmCPU.c:84), where the
 *     Z axis is ONE-WAY time tau in seconds: the traveltime of a zero-offset
 *     pair is 2*tau (psktmCPU.c:46, :78-79).
 *   - Trace layout: float[traceNo][tracePts], trace-contiguous
 *     (psktmCPU.c:85 reads traces[it + k*tracePts]).
 *   - Coordinates: midpoint and HALF-offset vectors, source = mid - off,
 *     receiver = mid + off (ktmConvertXYtoOffMid.m:12, psktmCPU.c:65-72).
 *   - "slowness" in the reference signature is a velocity v(tau) in m/s,
 *     one value per tau sample (psktmCPU.c:48 squares and inverts it).
 *   - Every int-returning entry point returns KTM_OK (0) or a KTM_ERR_* code;
 *     the void drop-ins record their status for ktmGetLastError().
 */
#ifndef KTM_H
#define KTM_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One image axis: axis[i] = imageStart + (float)i * imageStep.
 * Field names from psktmFunctions.c:10-14 and psktmCUDA.cu:226-237; the
 * reference defines no struct, so the field order is this library's. */
struct imageGrid {
    int   imagePnts;
    float imageStep;
    float imageStart;
};

/* Trace block description.  Field names from psktmCPU.c:29,59,82 and
 * psktmCUDA.cu:245-247; traceSampleRate is the sample interval in seconds. */
struct jobParams {
    int   traceNo;
    int   tracePts;
    float traceSampleRate;
};

/* ------------------------------------------------------------------------ */
/* Drop-in entry points (host buffers, synchronous, image overwritten)      */
/* ------------------------------------------------------------------------ */

/* Replaces ktmMigrationCPU, psktmCPU.c:13-23.  Same arguments, same result:
 * the image is bit-identical to psktmCPU.c run with one thread (the reference
 * loop races on image[] with more, psktmCPU.c:56-85).  Runs on the current
 * CUDA device. */
void ktmMigrationCPU(struct imageGrid* imageX, struct imageGrid* imageY,
                     struct imageGrid* imageZ, struct jobParams* config,
                     float* midX, float* midY, float* offX, float* offY,
                     float* traces, float* slowness, float* image);

/* Replaces ktmMigrationGPU, psktmCUDA.cu:211-221 (same signature as above).
 * Unlike the reference GPU host it has no Nx*Ny block limit (:298-301), no
 * traceNo % THREADS_X requirement (:95) and no Nz <= 2048 cap (:21-22). */
void ktmMigrationGPU(struct imageGrid* imageX, struct imageGrid* imageY,
                     struct imageGrid* imageZ, struct jobParams* config,
                     float* midX, float* midY, float* offX, float* offY,
                     float* traces, float* slowness, float* image);

/* psktmFunctions.c:19-39 and :1-17 (host helpers, same arithmetic). */
void initThreeAxes(struct imageGrid* imageX, struct imageGrid* imageY,
                   struct imageGrid* imageZ, float* imageXX, float* imageYY,
                   float* imageZZ);
void initTwoAxes(struct imageGrid* imageY, struct imageGrid* imageZ,
                 float* imageYY, float* imageZZ);

/* ------------------------------------------------------------------------ */
/* Status                                                                   */
/* ------------------------------------------------------------------------ */

enum {
    KTM_OK = 0,
    KTM_ERR_ARG = 1,        /* invalid argument (NULL pointer, bad size, bad enum) */
    KTM_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    KTM_ERR_NOMEM = 3,      /* device or host allocation failed */
    KTM_ERR_LIMIT = 4,      /* size beyond a documented kernel limit */
    KTM_ERR_IO = 5,         /* file could not be opened / read / written */
    KTM_ERR_TIMEOUT = 6,    /* a bounded device-side wait gave up */
    KTM_ERR_NODEVICE = 7    /* no CUDA device visible */
};

/* Status of the most recent call made by this host thread. */
int ktmGetLastError(void);
/* Human-readable message for the most recent failure of this host thread. */
const char* ktmGetLastErrorMessage(void);
const char* ktmGetErrorString(int code);

/* ------------------------------------------------------------------------ */
/* Extended migration job                                                   */
/* ------------------------------------------------------------------------ */

/* Kernel family. */
enum {
    KTM_MODE_REFERENCE = 0, /* psktmCPU.c arithmetic, bit-exact: F32 traces,
                               truncating pick, no aperture, 1-D velocity */
    KTM_MODE_FAST = 1,      /* SFU square roots, linear or truncating pick,
                               aperture, Vrms cube, F32/F16/BF16 traces */
    KTM_MODE_F64 = 2        /* FP64 arithmetic (accuracy reference on device) */
};

/* Trace sample formats. */
enum {
    KTM_FMT_F32 = 0,
    KTM_FMT_F16 = 1,        /* IEEE half, multiplied by a per-trace FP32 scale */
    KTM_FMT_BF16 = 2,       /* bfloat16, multiplied by a per-trace FP32 scale */
    KTM_FMT_IBM32 = 3,      /* IBM System/360 single precision words (inputData.bin,
                               ioFunctions.c:4-40): raw traces only, converted on the
                               device before filtering and packing */
    KTM_FMT_F64 = 4         /* double: raw traces of ktmMigrateColumnsF64 only (an FP64
                               pipeline's reference image); rejected elsewhere */
};

/* Sample pick. */
enum {
    KTM_PICK_TRUNCATE = 0,  /* it = (int)(t/dt), used when 0 < it < tracePts (psktmCPU.c:80-82) */
    KTM_PICK_LINEAR = 1     /* linear interpolation between samples; samples
                               outside 0 < j < tracePts read as zero */
};

typedef struct ktm_job {
    struct imageGrid imageX, imageY, imageZ;   /* Z = one-way tau, s */
    struct jobParams config;                   /* traceNo, tracePts, traceSampleRate */
    const float* midX;                         /* [traceNo] */
    const float* midY;
    const float* offX;                         /* half offsets */
    const float* offY;
    const void*  traces;                       /* [traceNo][traceStride] in traceFormat */
    const float* traceScale;                   /* [traceNo] multiplier (NULL: 1.0) */
    int   traceFormat;                         /* KTM_FMT_* (IBM32: raw traces only) */
    int   traceStride;                         /* samples between traces; 0 = tracePts */
    int   tracesPacked;                        /* 1: traces come from ktmPrepareTraces
                                                  (traceStride = its pitch, zero guard
                                                  samples at 0 and >= tracePts) */
    int   tracesPrefolded;                     /* 1: packed samples carry sqrt(j*dt)
                                                  (ktmPrepareTraces prefold = 1) */
    const float* velocity;                     /* m/s: [Nz], or [Nx][Ny][Nz] if velocityCube */
    int   velocityCube;
    float* image;                              /* [Nx][Ny][Nz] */
    int   mode;                                /* KTM_MODE_* */
    int   pick;                                /* KTM_PICK_* */
    float aperture;                            /* max |mid - x| in metres; <= 0: off */
    int   accumulate;                          /* 0: image overwritten, 1: added to */
    int   deviceMemory;                        /* 1: every pointer is device memory;
                                                  0: host memory, copied in and out */
    void* stream;                              /* cudaStream_t (NULL: legacy default) */
    int   tileRun;                             /* FAST mode: tau samples per warp run, 256,
                                                  384 or 512 (0: the run wasting the fewest
                                                  samples of Nz) */
    int   tileCols;                            /* FAST mode: image columns per CTA, one per
                                                  warp: 24 (one CTA per SM, the default for
                                                  0), 12 (two) or 8 (three); 12 and 8 serve the
                                                  linear pick with the prefolded or table
                                                  weight.  ktmAutotuneTile chooses these. */
    unsigned long long* pairsEvaluated;        /* optional device counter: pairs the
                                                  kernel evaluated (after culling) */
    /* FAST mode with raw (not packed) traces: the library prepares them first */
    int   rho;                                 /* KTM_RHO_* pre-filter (ktmApplyRhoFilter.m) */
    int   packFormat;                          /* KTM_FMT_* of the packed samples */
    int   weightMethod;                        /* KTM_WEIGHT_*: how FAST mode evaluates the
                                                  sqrt(t) of the weight when the samples
                                                  do not carry it */
    int   tileChunk;                           /* FAST mode: traces staged per shared-memory
                                                  chunk at most (0: as many as fit, <= 32) */
} ktm_job;

/* sqrt(t) of the reference weight t*sqrt(tau^2/t) = |tau| sqrt(t) (psktmCPU.c:85). */
enum {
    KTM_WEIGHT_TABLE = 0,   /* sqrt(j*dt) table interpolated at t/dt (relative error
                               ~1/(32 j^2)) -- two special-function ops per pair */
    KTM_WEIGHT_SQRT = 1,    /* sqrt.approx per pair -- three special-function ops */
    KTM_WEIGHT_PREFOLD = 2  /* ktmMigrate prepares raw traces with sqrt(j*dt) folded into
                               the samples (ktm_prep.prefold = 1): no weight work per pair.
                               Interpolating the product instead of the factors differs
                               from the reference weight by f(1-f) dg dd per pick (about
                               1e-4 relative L2 on deep images, up to ~6e-4 on shallow
                               ones); linear pick only.  Packed traces must have been
                               prepared with prefold = 1 (tracesPrefolded). */
};

/* Zero-initialise a job and fill in defaults (mode FAST, pick LINEAR, F32,
 * overwrite, host memory, tuned tiles). */
void ktmJobInit(ktm_job* job);

/* sizeof(ktm_job) as compiled into the library, for bindings (ctypes, cgo)
 * that lay the struct out themselves.  No counterpart in the reference. */
size_t ktmJobStructSize(void);

/* Run one migration.  Asynchronous on job->stream when deviceMemory = 1;
 * synchronous when host buffers are given.  Replaces the body of
 * ktmMigrationCPU (psktmCPU.c:56-90) with the extended method. */
int ktmMigrate(const ktm_job* job);

/* ------------------------------------------------------------------------ */
/* Trace preparation: rho pre-filter, weight fold, quantisation, packing    */
/* ------------------------------------------------------------------------ */

/* Rho filter options of ktmApplyRhoFilter.m (:39-58). */
enum {
    KTM_RHO_NONE = 0,
    KTM_RHO_2D = 1,         /* |omega| */
    KTM_RHO_25D = 2,        /* sqrt|omega| exp(i pi/4 sign omega) */
    KTM_RHO_3D = 3          /* i omega */
};

typedef struct ktm_prep {
    int   traceNo, tracePts;
    int   inStride;            /* samples between input traces (0: tracePts) */
    float sampleRate;          /* s */
    const float* in;           /* [traceNo][inStride] in inFormat, device memory */
    int   rho;                 /* KTM_RHO_*: the rho filter of ktmApplyRhoFilter.m:22-62
                                  (FFT length 2^ceil(log2 tracePts), omega = 2 pi k / dt
                                  with the script's scaling), applied per trace */
    int   rhoScriptOrder;      /* 1: also reproduce the script's trace rotation for an odd
                                  traceNo (Octave fftshift of a matrix shifts the trace
                                  axis too): output trace q = filtered input (q+1) mod n */
    int   prefold;             /* 1: multiply sample j by sqrt(j*dt) (the migration weight
                                  sqrt(t), moved from every pair to every sample) */
    int   outFormat;           /* KTM_FMT_F32 / F16 / BF16 */
    int   outPitch;            /* elements per packed trace (0: ktmPackedPitch) */
    void* out;                 /* [traceNo][outPitch], device memory, 16-byte aligned */
    float* outScale;           /* [traceNo] per-trace scale, device memory */
    void* stream;              /* cudaStream_t */
    int   inFormat;            /* KTM_FMT_F32 (0) or KTM_FMT_IBM32: IBM words converted as
                                  ktmIBM32toIEEE does, in the same pass */
} ktm_prep;

/* Default pitch of a packed trace: tracePts + 2 rounded up to 16 bytes. */
int ktmPackedPitch(int tracePts, int format);

/* Filter (optional), weight (optional), quantise and pack traces for the fast
 * migration kernel.  Packed trace k holds out[k][j] = q_j for 0 < j < tracePts
 * and zero at j = 0 and j >= tracePts (the reference's pick window 0 < it <
 * tracePts, psktmCPU.c:82); x_j = outScale[k] * q_j.  F16/BF16 scales put the
 * largest |sample| of each trace at 32768 / 1.  Replaces the Octave
 * pre-processing ktmApplyRhoFilter.m with a device step.  Asynchronous. */
int ktmPrepareTraces(const ktm_prep* prep);

/* ------------------------------------------------------------------------ */
/* Adjoint, velocity gradient, least-squares migration                      */
/* (no counterpart in the reference: it has no adjoint and no inversion)    */
/* ------------------------------------------------------------------------ */

/* Kirchhoff demigration, the exact transpose of ktmMigrate in FAST mode
 * (linear or truncating pick, KTM_WEIGHT_TABLE or KTM_WEIGHT_SQRT, aperture,
 * Vrms): reads the model from job->image [Nx][Ny][Nz] and writes
 *   data[k][j] = sum_p w(p,k) coef_j(t(p,k)/dt) m[p],   0 < j < tracePts,
 * into the packed F32 layout [traceNo][dataPitch] (dataPitch >= tracePts + 2,
 * a multiple of 4; zero guard samples), overwritten unless job->accumulate.
 * KTM_WEIGHT_PREFOLD (linear pick): the transpose of migrating samples
 * prefolded with sqrt(j*dt), w(p,k) = |tau_p| and every data[k][j] multiplied
 * by sqrt(j*dt) -- no weight work per pair.
 * job->traces is not read.  Device memory, asynchronous on job->stream. */
int ktmDemigrate(const ktm_job* job, float* data, int dataPitch);

/* Sensitivity of the migrated image to the RMS velocity at each image sample:
 * grad[p] = dI[p] / dv[p] for the job's packed traces (linear pick; table
 * weight or prefolded samples) -- the traveltime (and weight) derivative of
 * every pair, d/dv of t = sqrt(tau^2 + |s-x|^2/v^2) + sqrt(tau^2 + |r-x|^2/v^2).
 * For an objective J(I), dJ/dv[p] = dJ/dI[p] * grad[p].  grad is
 * [Nx][Ny][Nz], device memory; asynchronous. */
int ktmVrmsGradient(const ktm_job* job, float* grad);

/* Least-squares migration by conjugate gradients on the normal equations
 * (CGLS): minimise || L m - d ||^2, L = ktmDemigrate, L^T = ktmMigrate (FAST
 * mode, packed F32 traces).  All vectors and scalars stay on the device; the
 * CG dot products and norms are FP64.  With useGraph = 1 one iteration is
 * captured in a CUDA graph and replayed.  job.weightMethod = KTM_WEIGHT_PREFOLD
 * (linear pick) uses the prefolded operator pair: the residual is folded with
 * sqrt(j*dt) before each migration (one more data-sized workspace vector). */
typedef struct ktm_lsm {
    ktm_job job;                 /* geometry, coordinates, velocity, pick, aperture,
                                    weightMethod, stream; device memory */
    const float* data;           /* observed data, packed F32 [traceNo][dataPitch] */
    int   dataPitch;
    float* model;                /* [Nx][Ny][Nz]: starting model in, solution out */
    int   iterations;
    int   useGraph;
    double* residualNorms;       /* host [iterations+1]: ||d - L m_i|| (may be NULL) */
    double* gradientNorms;       /* host [iterations+1]: ||L^T (d - L m_i)|| (may be NULL) */
} ktm_lsm;
int ktmLeastSquaresMigrate(const ktm_lsm* lsm);

/* ------------------------------------------------------------------------ */
/* Batched target-oriented migration and tile tuning                        */
/* (no counterpart in the reference)                                        */
/* ------------------------------------------------------------------------ */

/* Many independent jobs (image patches of any size, trace sets of any size) in
 * ONE persistent launch: a queue of (job, 8 image columns, tau run, trace slice)
 * tiles sorted longest first, pulled by one CTA per SM slot.  Every job: FAST
 * mode, device memory, a packed trace set; all jobs share the trace format,
 * pick and weight, and the first job's tileRun (0: chosen from the jobs' Nz).
 * Images are overwritten.  Asynchronous on `stream`. */
int ktmMigrateBatch(const ktm_job* jobs, int njobs, void* stream);

/* Tile shape of the fast kernel (ktm_job.tileRun / tileCols / tileChunk).  The
 * reference's GPU kernel fixes its tile at compile time (THREADS_X x THREADS_Y,
 * psktmCUDA.cu:95-106); here it is chosen per job shape. */
typedef struct ktm_tile {
    int   tileRun;       /* tau samples per warp run: 512, 384 or 256 */
    int   tileCols;      /* image columns per CTA (one per warp): 24, 12 or 8 */
    int   tileChunk;     /* traces per shared-memory chunk at most (0: as many as fit) */
    int   ctasPerSm;     /* CTAs of that shape resident per SM: 1, 2 or 3 (24 warps) */
    float ms;            /* ktmAutotuneTile: one launch's time on the tuning sample */
} ktm_tile;

/* The candidate tiles of a job: tau runs 512 / 384 / 256 x CTA shapes (24, 12
 * or 8 columns per CTA where the job's path is built for them -- linear pick with
 * the prefolded or table weight -- else 24) x chunks (as many traces as fit, or
 * at most 8).  Writes up to `capacity` of them and their number to *count.
 * No device work.  No counterpart in the reference. */
int ktmTileCandidates(const ktm_job* job, ktm_tile* out, int capacity, int* count);

/* Tile tuning: times every candidate of ktmTileCandidates on up to 4096 of the
 * job's traces (a warm-up and two timed launches each) and returns the fastest in
 * *best (remembered per image / trace shape, format, pick and weight for the
 * process).  Overwrites job->image.  Device memory, packed traces; synchronous.
 * No counterpart in the reference. */
int ktmAutotuneTile(const ktm_job* job, ktm_tile* best);

/* ktmAutotuneTile, returning only the chosen tau run (the whole tile is
 * remembered the same way). */
int ktmAutotune(const ktm_job* job, int* tileRun);

/* ktmMigrate for callers that cannot allocate device memory while they run:
 * a processing loop that must never let cudaMalloc / cudaFree synchronise the
 * device, or a host framework that has already shared the GPU's memory out
 * among its own pools.  No counterpart in the reference.
 *   - Takes FAST mode, device memory and a packed trace set (ktmPrepareTraces);
 *     the caller passes every input and the output image as usual.
 *   - Calls no cudaMalloc, cudaFree or allocating routine.  Its only scratch,
 *     the partial images of the trace slices, is a static 16 MiB device array
 *     (4 Mi floats) that each GPU loading the library keeps until exit.
 *   - Limit: images of at most 2 Mi samples (Nx*Ny*Nz <= 2097152); larger
 *     images are rejected with KTM_ERR_LIMIT.
 *   - Accepts what ktmMigrateBatch accepts for one job: F32 / F16 / BF16 packed
 *     samples, linear or truncating pick, KTM_WEIGHT_TABLE / _SQRT, and
 *     KTM_WEIGHT_PREFOLD with samples prepared with prefold = 1; accumulate.
 *   - The first call on a device looks up that device's copy of the array
 *     (with the device current).  Under CUDA's lazy module loading (the
 *     default) that first call also loads the module holding the array, which
 *     creates it on the device: a one-time implicit allocation that may
 *     synchronise.  Make that first call during set-up, before any stream
 *     capture.
 *   - Every call uses the same array: calls that overlap on the GPU (other
 *     streams, other host threads on the same device) race.  Nothing in the
 *     array has to start at zero; each call writes every partial image before
 *     it reads it.  After KTM_ERR_TIMEOUT from ktmCheckDeviceWaits the image
 *     of the call concerned is undefined (a tile that gave up wrote nothing). */
int ktmMigratePackedNoAlloc(const ktm_job* job);

/* FP64 device evaluation of the job's method (pick, aperture, Vrms cube,
 * weight) for the image columns columns[0..ncols) (column index = ix*Ny + iy;
 * columns == NULL: 0..ncols-1): out[q][Nz].  Device memory only.  Used to
 * measure the error of the FP32 / FP16 / BF16 paths on images too large for a
 * CPU evaluation.  No counterpart in the reference. */
int ktmMigrateColumnsF64(const ktm_job* job, const int* columns, int ncols, double* out);

/* ------------------------------------------------------------------------ */
/* The reference's data formats (host code, no device needed)               */
/* ------------------------------------------------------------------------ */

/* inp.txt: 12 space-separated numbers (ktmVisualizeOutputFile.m:22-48,
 * ktmWriteTraceBlockConstOffset.m:154-167): tracePts, dt [s], traceNo,
 * x start/step/points, y start/step/points, tau start/step/points. */
typedef struct ktm_inp {
    int   tracePts;
    float sampleRate;          /* s */
    int   traceNo;
    struct imageGrid x, y, z;
} ktm_inp;
int ktmReadInp(const char* path, ktm_inp* inp);
int ktmWriteInp(const char* path, const ktm_inp* inp);   /* same layout, "%f " per value */

/* The survey of one data directory (loadInputData, ioFunctions.c:94-153):
 * inputData.bin (traceNo x tracePts uint32 IBM-32 words when dataIsIBM, or
 * float32 for the writers' impulse option), inputSrcX/Y.bin and inputRecX/Y.bin (float32
 * [traceNo]), velModel.bin (float32 [Nz] or [Nx][Ny][Nz]).  Coordinates become
 * midpoints and half offsets (ktmConvertXYtoOffMid.m:12) in FP64; with
 * rebase = 1 they and the image axes are shifted by the survey origin (the
 * smallest source/receiver x and y) before rounding to float.  Buffers are
 * malloc'd; release them with ktmFreeSurvey. */
typedef struct ktm_survey {
    ktm_inp inp;
    void* traces;              /* [traceNo][tracePts] 4-byte words in traceFormat */
    int   traceFormat;         /* KTM_FMT_IBM32 or KTM_FMT_F32, as read: the words stay
                                  unconverted for the device (ktm_job.traceFormat) */
    float *midX, *midY, *offX, *offY;
    float* velocity;
    int   velocityCube;
    double originX, originY;   /* subtracted when rebased */
} ktm_survey;
int ktmLoadSurvey(const char* dir, int dataIsIBM, int rebase, ktm_survey* out);
void ktmFreeSurvey(ktm_survey* s);
/* velModel.bin (ktmWriteVelModel.m:22-23) for the grid of `inp`: the Nx*Ny*Nz cube
 * when the file holds exactly that many values, else its first Nz values (the
 * writer may have appended models).  *velocity is malloc'd (release with free). */
int ktmReadVelModel(const char* path, const ktm_inp* inp, float** velocity, int* velocityCube);
/* outputData.bin: float32 [Nx][Ny][Nz], tau fastest (ktmVisualizeOutputFile.m:16-28). */
int ktmWriteImage(const char* path, const float* image, size_t count);

/* The reference's file functions, same names, arguments and behaviour
 * (ioFunctions.c:44-153), for a caller written against ioFunctions.c.  The
 * reference uses struct fileInputPtrs without defining it (:96-148 name the
 * fields); the field order is this library's.  Each records its status for
 * ktmGetLastError(); ktmLoadSurvey is the checked replacement. */
struct fileInputPtrs {
    int   flag;            /* 1 when an input file could not be opened */
    FILE* inputData;
    FILE* inputSrcX;
    FILE* inputSrcY;
    FILE* inputRecX;
    FILE* inputRecY;
};
/* ioFunctions.c:44-56: whole 4-byte words from the current position to the end;
 * the file is left at its start. */
int fileSizeFourBytes(FILE* fin);
/* ioFunctions.c:60-76: n words from the current position into a new malloc'd
 * buffer (free it); the file is left at its start.  Words past the end of the
 * file read as zero here (uninitialised in the reference). */
unsigned int* binReadUints(FILE* fin, int n);
float* binReadFloats(FILE* fin, int n);
/* ioFunctions.c:79-83: t floats to fout. */
void fileWrite(FILE* fout, float* ptr, int t);
/* ioFunctions.c:87-90: prints "Can't open <str>." */
void errorMessage(char* str);
/* ioFunctions.c:94-153: opens ../data/inputData.bin, inputSrcX.bin, inputSrcY.bin,
 * inputRecX.bin and inputRecY.bin (relative to the working directory, mode "r+b");
 * flag = 1 and a message on stdout for each that cannot be opened. */
void loadInputData(struct fileInputPtrs* input);

/* ioFunctions.c:4-40 (same name and arguments): IBM-32 words to IEEE float,
 * sign * (fraction / 0xFFFFFF) * 16^(exponent - 64), on the current device
 * (host buffers, synchronous).  Bit-identical to the reference. */
void ktmIBM32toIEEE(unsigned int* input, float* output, int n);
/* The same conversion on device buffers, asynchronous on `stream`. */
int ktmIBM32toIEEEDevice(const unsigned int* input, float* output, size_t n, void* stream);

/* SEG-Y files (rev 0 layout), the C replacement of ktmGetInputMeta.m:21-150 and
 * ktmGetInputTrace.m:29-75.  Big-endian fields (the standard) unless bigEndian = 0.
 * Trace-header fields are decoded as signed two's-complement numbers (the scripts'
 * int32()/int16() casts saturate negative values instead). */
typedef struct ktm_segy_info {
    char text[3240];                /* the EBCDIC reel header as ASCII, 40 lines of 80
                                       characters, '\n'-separated; the characters the
                                       script's table maps (ktmGetInputMeta.m:30-45),
                                       '?' for the rest */
    unsigned int reel32[3];         /* job, line, reel numbers (bytes 3201-3212) */
    unsigned int reel16[24];        /* the 16-bit binary reel header fields (3213-3260),
                                       in the order ktmListInputMeta.m names them */
    int   sampleInterval;           /* us (reel16[2]) */
    int   samplesPerTrace;          /* reel16[4] */
    int   format;                   /* reel16[6]: 1 IBM, 2 int32, 3 int16, 5 IEEE, 8 int8 */
    int   bigEndian;
    long long traceBytes;           /* 240 + samples * bytes per sample */
    long long traceCount;           /* whole traces in the file */
} ktm_segy_info;

typedef struct ktm_segy_trace {
    int    values[101];             /* the 240-byte header as ktmGetInputMeta.m:132 groups
                                       it: 7 int32 (bytes 1-28), 4 int16 (29-36), 8 int32
                                       (37-68), 2 int16 (69-72, [20] = coordinate scalar),
                                       4 int32 (73-88: [21..24] source x, y, receiver x, y),
                                       76 int16 (89-240) */
    double srcX, srcY, recX, recY;  /* coordinates with the scalar applied
                                       (> 0 multiplier, < 0 divisor, 0 = 1) */
} ktm_segy_trace;

/* Read the reel headers; the trace count follows from the file size. */
int ktmSegyOpen(const char* path, int bigEndian, ktm_segy_info* info);
/* Traces [first, first + count): samples into `samples` ([count][samplesPerTrace]
 * 4-byte words: IBM words as stored for format 1 -- KTM_FMT_IBM32, decoded on the
 * GPU -- and float for the other formats) and/or headers (either may be NULL). */
int ktmSegyReadTraces(const char* path, const ktm_segy_info* info, long long first,
                      long long count, void* samples, ktm_segy_trace* headers);
/* KTM_FMT_IBM32 for format 1, KTM_FMT_F32 otherwise (the words ktmSegyReadTraces writes). */
int ktmSegyTraceFormat(const ktm_segy_info* info);
/* A survey from traces [first, first + count) of a SEG-Y file (count < 0: to the end):
 * samples as ktmSegyReadTraces writes them, midpoints / half offsets from the scaled
 * source and receiver coordinates in FP64 (ktmConvertXYtoOffMid.m:12; rebase = 1
 * subtracts the survey origin first), tracePts and sampleRate from the reel header.
 * SEG-Y carries no image grid or velocity: inp.x/y/z and velocity are left zero for
 * the caller (subtract originX / originY from the x / y starts when rebased).
 * Release with ktmFreeSurvey. */
int ktmLoadSegySurvey(const char* path, int bigEndian, long long first, long long count,
                      int rebase, ktm_survey* out);

/* ------------------------------------------------------------------------ */
/* Time-axis interpolation (ktmInterpTraceBlock.m:134-154, opt 2)           */
/* ------------------------------------------------------------------------ */

typedef struct ktm_interp {
    int   traceNo, tracePts;
    int   levels;                   /* N: 2^N output samples per input interval (0..10) */
    const float* in;                /* [traceNo][inStride], device memory */
    int   inStride;                 /* 0: tracePts */
    float* out;                     /* [traceNo][outStride], device memory */
    long long outStride;            /* 0: ktmInterpLength(tracePts, levels) */
    void* stream;                   /* cudaStream_t */
} ktm_interp;

/* Samples after interpolation: (tracePts - 1) * 2^levels + 1 (0 for no samples). */
long long ktmInterpLength(int tracePts, int levels);
/* Linear interpolation of every trace onto t = j / 2^levels (the new sample
 * interval is dt / 2^levels), evaluated in FP64 as Octave's interp1 does and
 * rounded to float: bit-identical to the script on float input.  Asynchronous. */
int ktmInterpTraces(const ktm_interp* interp);

/* The library keeps its temporary device memory (the device copies of host-memory
 * jobs, packing buffers, trace-slice partial images, the least-squares workspace)
 * in a memory pool of its own per device that holds on to freed memory, so
 * repeated calls do not map memory again.  This returns that memory to the
 * device; it synchronises every device the library has used.  No counterpart in
 * the reference. */
int ktmReleaseMemory(void);

/* Counters of that memory pool: *allocations = stream-ordered allocations the
 * library has made since it was loaded (all devices); *reservedBytes /
 * *usedBytes = the current device's pool, reserved and in use (0 when the
 * library has not allocated on it).  Any pointer may be NULL.  No counterpart
 * in the reference. */
int ktmMemoryStats(unsigned long long* allocations, size_t* reservedBytes, size_t* usedBytes);

/* The fast kernels stage each chunk of packed trace rows into shared memory with
 * one bulk (TMA) copy and wait for it with a bound of one second.  A wait that
 * runs out ends its tile without output and is counted on the device.  This
 * synchronises the current device and returns KTM_ERR_TIMEOUT (resetting the
 * count) when any such wait ran out since the last check, else KTM_OK.  The
 * images of the calls since the last check are then undefined: a tile that
 * gave up contributed nothing, and where the launch sums trace slices, the
 * slice it left unwritten holds stale values.  The
 * synchronous entry points (host-memory ktmMigrate, ktmLeastSquaresMigrate)
 * check by themselves; after asynchronous calls check at the caller's own
 * synchronisation point.  No counterpart in the reference. */
int ktmCheckDeviceWaits(void);

/* Self-test of that mechanism on the current device: one CTA bulk-copies 64 KiB
 * into shared memory and checks the bytes; with stall = 1 it first waits on a
 * barrier that nothing arrives on, which gives up after limitMs (1..10000).
 * Synchronous; returns ktmCheckDeviceWaits()'s status: KTM_ERR_TIMEOUT for
 * stall = 1, KTM_OK for stall = 0. */
int ktmSelfTestDeviceWait(int stall, int limitMs);

/* ------------------------------------------------------------------------ */
/* Synthetic data and measurement                                           */
/* ------------------------------------------------------------------------ */

/* Seeded synthetic traces on the device: out[k][j] = sum over scatterers s of
 * amp_s * Ricker(j*dt - t_ks) + noise * N(0,1), t_ks the double-square-root
 * time source -> scatterer -> receiver with the scatterer's RMS velocity.
 * scatterers = double[scatterNo][5] (x, y, tau0, v, amplitude).  The noise is
 * a counter hash of (seed, traceOffset + k, j), identical to the numpy
 * generator of the Python package.  All pointers device memory; asynchronous.
 * Stands in for field data (the reference's impulse option,
 * ktmWriteTraceBlockConstOffset.m:65-83, is the closest counterpart). */
int ktmSynthesizeTraces(int traceNo, int tracePts, float sampleRate, const float* midX,
                        const float* midY, const float* offX, const float* offY,
                        int scatterNo, const double* scatterers, double freq, double noise,
                        unsigned long long seed, int traceOffset, float* out, void* stream);

/* ------------------------------------------------------------------------ */
/* Measurement                                                              */
/* ------------------------------------------------------------------------ */

/* Pipe throughput of the current GPU, measured now: sqrt.approx.f32 and
 * rsqrt.approx.f32 results per second (the special-function unit that bounds
 * the migration kernel) and FP32 FMAs per second.  Any pointer may be NULL.
 * Synchronous.  No counterpart in the reference. */
int ktmProbePeaks(double* sqrtPerSec, double* rsqrtPerSec, double* ffmaPerSec);

#ifdef __cplusplus
}
#endif
#endif /* KTM_H */
