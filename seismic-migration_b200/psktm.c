/*
 * psktm -- migrate one data directory written by the reference's Octave
 * writers (ktmWriteTraceBlockConstOffset.m, ktmWriteVelModel.m) and write
 * outputData.bin for ktmVisualizeOutputFile.m.  The reference has no such
 * driver: its C side stops at loadInputData (ioFunctions.c:94-153) and
 * ktmMigrationCPU (psktmCPU.c:13); this is the program those pieces imply.
 *
 *   psktm [options] DATA_DIR
 *
 *   --float              inputData.bin holds float32 (the writers' impulse
 *                        option, ktmWriteTraceBlockConstOffset.m:145); the
 *                        default is IBM-32 words (:142), converted on the GPU
 *   --segy FILE          traces, coordinates (coordinate scalar applied) and the
 *                        sample interval from a SEG-Y file instead of
 *                        inputData.bin / inputSrc* / inputRec*; DATA_DIR still
 *                        gives the image grid (inp.txt) and velModel.bin
 *   --le                 the SEG-Y file is little-endian
 *   --mode reference     psktmCPU.c arithmetic, bit-identical (default)
 *   --mode fast          the fast kernel (linear pick, FP16 samples, ...)
 *   --pick linear|truncate        fast mode (default linear)
 *   --format f32|f16|bf16         fast mode sample format (default f16)
 *   --rho none|2d|2.5d|3d         fast mode rho pre-filter (default none)
 *   --aperture METRES             fast mode midpoint aperture (default off)
 *   --rebase | --no-rebase        shift coordinates and image axes by the survey
 *                        origin (in FP64) before rounding to float; default on
 *                        in fast mode, off in reference mode (bit-identity)
 *   -o FILE              output (default DATA_DIR/outputData.bin)
 *   -q                   quiet
 *
 * The GPU is the current CUDA device (select one with CUDA_VISIBLE_DEVICES).
 * Exit status: 0 on success, 1 on a usage error, 2 on a library error.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "ktm.h"

static void usage(const char* argv0)
{
    fprintf(stderr,
            "usage: %s [--float] [--segy FILE [--le]] [--mode reference|fast] [--pick linear|truncate]\n"
            "       [--format f32|f16|bf16] [--rho none|2d|2.5d|3d] [--aperture M]\n"
            "       [--rebase|--no-rebase] [-o FILE] [-q] DATA_DIR\n",
            argv0);
}

static int fail(const char* what)
{
    fprintf(stderr, "psktm: %s: %s (%s)\n", what, ktmGetLastErrorMessage(),
            ktmGetErrorString(ktmGetLastError()));
    return 2;
}

static double now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int main(int argc, char** argv)
{
    const char* dir = NULL;
    const char* outPath = NULL;
    const char* segy = NULL;
    int segyLE = 0;
    int isFloat = 0, mode = KTM_MODE_REFERENCE, pick = KTM_PICK_LINEAR, fmt = KTM_FMT_F16;
    int rho = KTM_RHO_NONE, rebase = -1, quiet = 0;
    float aperture = 0.0f;
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        const char* v = i + 1 < argc ? argv[i + 1] : NULL;
        if (!strcmp(a, "--float")) {
            isFloat = 1;
        } else if (!strcmp(a, "--le")) {
            segyLE = 1;
        } else if (v && !strcmp(a, "--segy")) {
            segy = v;
            i++;
        } else if (!strcmp(a, "--rebase")) {
            rebase = 1;
        } else if (!strcmp(a, "--no-rebase")) {
            rebase = 0;
        } else if (!strcmp(a, "-q")) {
            quiet = 1;
        } else if (!strcmp(a, "-h") || !strcmp(a, "--help")) {
            usage(argv[0]);
            return 0;
        } else if (v && !strcmp(a, "--mode")) {
            if (!strcmp(v, "reference")) mode = KTM_MODE_REFERENCE;
            else if (!strcmp(v, "fast")) mode = KTM_MODE_FAST;
            else { usage(argv[0]); return 1; }
            i++;
        } else if (v && !strcmp(a, "--pick")) {
            if (!strcmp(v, "linear")) pick = KTM_PICK_LINEAR;
            else if (!strcmp(v, "truncate")) pick = KTM_PICK_TRUNCATE;
            else { usage(argv[0]); return 1; }
            i++;
        } else if (v && !strcmp(a, "--format")) {
            if (!strcmp(v, "f32")) fmt = KTM_FMT_F32;
            else if (!strcmp(v, "f16")) fmt = KTM_FMT_F16;
            else if (!strcmp(v, "bf16")) fmt = KTM_FMT_BF16;
            else { usage(argv[0]); return 1; }
            i++;
        } else if (v && !strcmp(a, "--rho")) {
            if (!strcmp(v, "none")) rho = KTM_RHO_NONE;
            else if (!strcmp(v, "2d")) rho = KTM_RHO_2D;
            else if (!strcmp(v, "2.5d")) rho = KTM_RHO_25D;
            else if (!strcmp(v, "3d")) rho = KTM_RHO_3D;
            else { usage(argv[0]); return 1; }
            i++;
        } else if (v && !strcmp(a, "--aperture")) {
            aperture = (float)atof(v);
            i++;
        } else if (v && !strcmp(a, "-o")) {
            outPath = v;
            i++;
        } else if (a[0] == '-' || dir) {
            usage(argv[0]);
            return 1;
        } else {
            dir = a;
        }
    }
    if (!dir) {
        usage(argv[0]);
        return 1;
    }
    if (rebase < 0) rebase = mode == KTM_MODE_FAST;
    char defOut[4096];
    if (!outPath) {
        snprintf(defOut, sizeof(defOut), "%s/outputData.bin", dir);
        outPath = defOut;
    }

    const double t0 = now();
    ktm_survey sv;
    if (!segy) {
        if (ktmLoadSurvey(dir, !isFloat, rebase, &sv)) return fail("reading the survey");
    } else {
        char path[4096];
        ktm_inp grid;
        snprintf(path, sizeof(path), "%s/inp.txt", dir);
        if (ktmReadInp(path, &grid)) return fail("reading inp.txt");
        if (ktmLoadSegySurvey(segy, !segyLE, 0, -1, rebase, &sv)) return fail("reading the SEG-Y file");
        sv.inp.x = grid.x;
        sv.inp.y = grid.y;
        sv.inp.z = grid.z;
        sv.inp.x.imageStart = (float)((double)grid.x.imageStart - sv.originX);
        sv.inp.y.imageStart = (float)((double)grid.y.imageStart - sv.originY);
        snprintf(path, sizeof(path), "%s/velModel.bin", dir);
        if (ktmReadVelModel(path, &sv.inp, &sv.velocity, &sv.velocityCube)) {
            ktmFreeSurvey(&sv);
            return fail("reading velModel.bin");
        }
    }
    const double t1 = now();

    const size_t nimg = (size_t)sv.inp.x.imagePnts * sv.inp.y.imagePnts * sv.inp.z.imagePnts;
    float* image = (float*)malloc(nimg ? nimg * sizeof(float) : sizeof(float));
    if (!image) {
        ktmFreeSurvey(&sv);
        fprintf(stderr, "psktm: out of host memory for the image\n");
        return 2;
    }
    ktm_job job;
    ktmJobInit(&job);
    job.imageX = sv.inp.x;
    job.imageY = sv.inp.y;
    job.imageZ = sv.inp.z;
    job.config.traceNo = sv.inp.traceNo;
    job.config.tracePts = sv.inp.tracePts;
    job.config.traceSampleRate = sv.inp.sampleRate;
    job.midX = sv.midX;
    job.midY = sv.midY;
    job.offX = sv.offX;
    job.offY = sv.offY;
    job.traces = sv.traces;
    job.traceFormat = sv.traceFormat;
    job.velocity = sv.velocity;
    job.velocityCube = sv.velocityCube;
    job.image = image;
    job.mode = mode;
    job.deviceMemory = 0;
    if (mode == KTM_MODE_REFERENCE) {
        job.pick = KTM_PICK_TRUNCATE;
    } else {
        job.pick = pick;
        job.packFormat = fmt;
        job.rho = rho;
        job.aperture = aperture;
    }
    int rc = ktmMigrate(&job);
    const double t2 = now();
    if (rc) {
        free(image);
        ktmFreeSurvey(&sv);
        return fail("migration");
    }
    rc = ktmWriteImage(outPath, image, nimg);
    const double t3 = now();
    if (!quiet && !rc) {
        printf("psktm: %d traces x %d samples -> %d x %d x %d image (%s, %s%s) in %.3f s "
               "(read %.3f s, migrate %.3f s, write %.3f s) -> %s\n",
               sv.inp.traceNo, sv.inp.tracePts, sv.inp.x.imagePnts, sv.inp.y.imagePnts,
               sv.inp.z.imagePnts, mode == KTM_MODE_REFERENCE ? "reference" : "fast",
               sv.traceFormat == KTM_FMT_IBM32 ? "IBM-32 input" : "float input",
               rebase ? ", rebased" : "", t3 - t0, t1 - t0, t2 - t1, t3 - t2, outPath);
        if (rebase)
            printf("psktm: arithmetic relative to the survey origin x = %.3f, y = %.3f "
                   "(the image grid is the one inp.txt names)\n", sv.originX, sv.originY);
    }
    free(image);
    ktmFreeSurvey(&sv);
    if (rc) return fail("writing the image");
    return 0;
}
