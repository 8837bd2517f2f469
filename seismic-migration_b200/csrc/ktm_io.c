/*
 * ktm_io.c -- the reference's on-disk formats, host side of libktm.so.
 *
 *   inp.txt         12 numbers: tracePts, dt [s], traceNo, x start/step/points,
 *                   y start/step/points, tau start/step/points
 *                   (ktmVisualizeOutputFile.m:22-48; written by
 *                   ktmWriteTraceBlockConstOffset.m:154-167 with "%f ")
 *   inputData.bin   traceNo x tracePts 4-byte words, trace after trace: IBM-32
 *                   (the writers' default, :142) or float32 (impulse option, :145)
 *   inputSrcX.bin, inputSrcY.bin, inputRecX.bin, inputRecY.bin
 *                   float32 [traceNo] (:149-152)
 *   velModel.bin    float32 (ktmWriteVelModel.m:22-23): [Nz], or [Nx][Ny][Nz]
 *   outputData.bin  float32 [Nx][Ny][Nz], tau fastest (ktmVisualizeOutputFile.m:16-28)
 *
 * ktmLoadSurvey and the readers below replace loadInputData / binReadFloats /
 * binReadUints / fileWrite (ioFunctions.c:44-153): paths are given (not fixed
 * to ../data), sizes come from inp.txt and are checked against the file sizes,
 * and every failure returns KTM_ERR_IO with a message instead of printing.
 * The reference's own names and arguments are exported too, with its
 * behaviour, for a caller written against ioFunctions.c (end of this file).
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/ktm.h"

/* status of the calling thread, kept by ktm_api.cu */
int ktm_io_error(int code, const char* msg);
int ktm_io_ok(void);

static int io_fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return ktm_io_error(code, buf);
}

static long file_size(FILE* f)
{
    long cur = ftell(f);
    if (fseek(f, 0, SEEK_END) != 0) return -1;
    long n = ftell(f);
    fseek(f, cur, SEEK_SET);
    return n;
}

/* read exactly `count` 4-byte values from dir/name into a new buffer */
static int read_words(const char* dir, const char* name, size_t count, void** out, size_t* have)
{
    char path[4096];
    snprintf(path, sizeof(path), "%s/%s", dir, name);
    FILE* f = fopen(path, "rb");
    if (!f) return io_fail(KTM_ERR_IO, "cannot open %s", path);
    long bytes = file_size(f);
    if (bytes < 0) {
        fclose(f);
        return io_fail(KTM_ERR_IO, "cannot size %s", path);
    }
    if (have) *have = (size_t)bytes / 4;
    if (count == 0) count = (size_t)bytes / 4;
    if ((size_t)bytes < count * 4) {
        fclose(f);
        return io_fail(KTM_ERR_IO, "%s holds %ld bytes, %zu needed", path, bytes, count * 4);
    }
    void* buf = malloc(count * 4 > 0 ? count * 4 : 4);
    if (!buf) {
        fclose(f);
        return io_fail(KTM_ERR_NOMEM, "out of host memory reading %s", path);
    }
    size_t got = fread(buf, 4, count, f);
    fclose(f);
    if (got != count) {
        free(buf);
        return io_fail(KTM_ERR_IO, "short read of %s", path);
    }
    *out = buf;
    return KTM_OK;
}

int ktmReadInp(const char* path, ktm_inp* inp)
{
    if (!path || !inp) return io_fail(KTM_ERR_ARG, "NULL argument");
    FILE* f = fopen(path, "r");
    if (!f) return io_fail(KTM_ERR_IO, "cannot open %s", path);
    double c[12];
    int n = 0;
    while (n < 12 && fscanf(f, "%lf", &c[n]) == 1) n++;
    fclose(f);
    if (n != 12) return io_fail(KTM_ERR_IO, "%s: %d numbers, 12 expected", path, n);
    inp->tracePts = (int)lround(c[0]);
    inp->sampleRate = (float)c[1];
    inp->traceNo = (int)lround(c[2]);
    inp->x.imageStart = (float)c[3]; inp->x.imageStep = (float)c[4]; inp->x.imagePnts = (int)lround(c[5]);
    inp->y.imageStart = (float)c[6]; inp->y.imageStep = (float)c[7]; inp->y.imagePnts = (int)lround(c[8]);
    inp->z.imageStart = (float)c[9]; inp->z.imageStep = (float)c[10]; inp->z.imagePnts = (int)lround(c[11]);
    if (inp->tracePts < 0 || inp->traceNo < 0 || inp->x.imagePnts < 0 || inp->y.imagePnts < 0 ||
        inp->z.imagePnts < 0)
        return io_fail(KTM_ERR_IO, "%s: negative size", path);
    return ktm_io_ok();
}

int ktmWriteInp(const char* path, const ktm_inp* inp)
{
    if (!path || !inp) return io_fail(KTM_ERR_ARG, "NULL argument");
    FILE* f = fopen(path, "w");
    if (!f) return io_fail(KTM_ERR_IO, "cannot create %s", path);
    fprintf(f, "%f %f %f %f %f %f %f %f %f %f %f %f ", (double)inp->tracePts,
            (double)inp->sampleRate, (double)inp->traceNo, (double)inp->x.imageStart,
            (double)inp->x.imageStep, (double)inp->x.imagePnts, (double)inp->y.imageStart,
            (double)inp->y.imageStep, (double)inp->y.imagePnts, (double)inp->z.imageStart,
            (double)inp->z.imageStep, (double)inp->z.imagePnts);
    if (fclose(f) != 0) return io_fail(KTM_ERR_IO, "cannot write %s", path);
    return ktm_io_ok();
}

int ktmReadVelModel(const char* path, const ktm_inp* inp, float** velocity, int* velocityCube)
{
    if (!path || !inp || !velocity || !velocityCube) return io_fail(KTM_ERR_ARG, "NULL argument");
    *velocity = NULL;
    *velocityCube = 0;
    FILE* f = fopen(path, "rb");
    if (!f) return io_fail(KTM_ERR_IO, "cannot open %s", path);
    long bytes = file_size(f);
    fclose(f);
    if (bytes < 0) return io_fail(KTM_ERR_IO, "cannot size %s", path);
    const size_t nvel = (size_t)bytes / 4;
    const size_t nz = (size_t)inp->z.imagePnts;
    const size_t ncube = (size_t)inp->x.imagePnts * inp->y.imagePnts * nz;
    /* the cube when the file holds exactly Nx*Ny*Nz values (and that differs from Nz),
       else the first Nz values (ktmWriteVelModel.m may have appended models) */
    const int cube = nvel == ncube && ncube != nz;
    if (!cube && nvel < nz)
        return io_fail(KTM_ERR_IO, "%s holds %zu values; %zu (1-D) or %zu (cube) expected", path,
                       nvel, nz, ncube);
    const char* slash = strrchr(path, '/');
    char dir[4096];
    const char* name = path;
    if (slash) {
        snprintf(dir, sizeof(dir), "%.*s", (int)(slash - path), path);
        name = slash + 1;
    } else {
        snprintf(dir, sizeof(dir), ".");
    }
    void* v = NULL;
    const int rc = read_words(dir, name, cube ? ncube : nz, &v, NULL);
    if (rc) return rc;
    *velocity = (float*)v;
    *velocityCube = cube;
    return ktm_io_ok();
}

void ktmFreeSurvey(ktm_survey* s)
{
    if (!s) return;
    free(s->traces); free(s->midX); free(s->midY); free(s->offX); free(s->offY); free(s->velocity);
    memset(s, 0, sizeof(*s));
}

int ktmLoadSurvey(const char* dir, int dataIsIBM, int rebase, ktm_survey* out)
{
    if (!dir || !out) return io_fail(KTM_ERR_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    char path[4096];
    snprintf(path, sizeof(path), "%s/inp.txt", dir);
    int rc = ktmReadInp(path, &out->inp);
    if (rc) return rc;
    const size_t ntr = (size_t)out->inp.traceNo, nt = (size_t)out->inp.tracePts;
    void *data = NULL, *sx = NULL, *sy = NULL, *rx = NULL, *ry = NULL;
    float* vel = NULL;
    int cube = 0;
    snprintf(path, sizeof(path), "%s/velModel.bin", dir);
    if ((rc = read_words(dir, "inputData.bin", ntr * nt, &data, NULL)) ||
        (rc = read_words(dir, "inputSrcX.bin", ntr, &sx, NULL)) ||
        (rc = read_words(dir, "inputSrcY.bin", ntr, &sy, NULL)) ||
        (rc = read_words(dir, "inputRecX.bin", ntr, &rx, NULL)) ||
        (rc = read_words(dir, "inputRecY.bin", ntr, &ry, NULL)) ||
        (rc = ktmReadVelModel(path, &out->inp, &vel, &cube))) {
        free(data); free(sx); free(sy); free(rx); free(ry); free(vel);
        return rc;
    }
    out->velocityCube = cube;
    out->velocity = vel;
    out->traces = data;   /* IBM words stay as read: the device converts them */
    out->traceFormat = dataIsIBM ? KTM_FMT_IBM32 : KTM_FMT_F32;
    const float *Sx = (const float*)sx, *Sy = (const float*)sy, *Rx = (const float*)rx,
                *Ry = (const float*)ry;
    double ox = 0.0, oy = 0.0;
    if (rebase && ntr > 0) {
        ox = Sx[0]; oy = Sy[0];
        for (size_t k = 0; k < ntr; k++) {
            ox = fmin(ox, fmin((double)Sx[k], (double)Rx[k]));
            oy = fmin(oy, fmin((double)Sy[k], (double)Ry[k]));
        }
        ox = floor(ox);
        oy = floor(oy);
        out->inp.x.imageStart = (float)((double)out->inp.x.imageStart - ox);
        out->inp.y.imageStart = (float)((double)out->inp.y.imageStart - oy);
    }
    out->originX = ox;
    out->originY = oy;
    out->midX = (float*)malloc(ntr * 4 + 4);
    out->midY = (float*)malloc(ntr * 4 + 4);
    out->offX = (float*)malloc(ntr * 4 + 4);
    out->offY = (float*)malloc(ntr * 4 + 4);
    if (!out->midX || !out->midY || !out->offX || !out->offY) {
        free(sx); free(sy); free(rx); free(ry);
        ktmFreeSurvey(out);
        return io_fail(KTM_ERR_NOMEM, "out of host memory");
    }
    /* ktmConvertXYtoOffMid.m:12 in FP64: mid = (r + s)/2, off = (r - s)/2 */
    for (size_t k = 0; k < ntr; k++) {
        const double s_x = Sx[k], s_y = Sy[k], r_x = Rx[k], r_y = Ry[k];
        out->midX[k] = (float)((r_x + s_x) / 2.0 - ox);
        out->midY[k] = (float)((r_y + s_y) / 2.0 - oy);
        out->offX[k] = (float)((r_x - s_x) / 2.0);
        out->offY[k] = (float)((r_y - s_y) / 2.0);
    }
    free(sx); free(sy); free(rx); free(ry);
    return ktm_io_ok();
}

int ktmWriteImage(const char* path, const float* image, size_t count)
{
    if (!path || (!image && count)) return io_fail(KTM_ERR_ARG, "NULL argument");
    FILE* f = fopen(path, "wb");
    if (!f) return io_fail(KTM_ERR_IO, "cannot create %s", path);
    size_t put = fwrite(image, sizeof(float), count, f);
    int bad = fclose(f) != 0 || put != count;
    if (bad) return io_fail(KTM_ERR_IO, "cannot write %s", path);
    return ktm_io_ok();
}

/* ------------------------------------------------------------------------ */
/* The reference's file functions under its own names (ioFunctions.c:44-153) */
/* ------------------------------------------------------------------------ */

/* Whole 4-byte words from the current position to the end of the file
 * (ioFunctions.c:44-56 counts them by reading word after word; the size comes
 * from the file position here, with the same result), then back to the start. */
int fileSizeFourBytes(FILE* fin)
{
    if (!fin) return io_fail(KTM_ERR_ARG, "fileSizeFourBytes: NULL file"), -1;
    long words = -1;
    const long cur = ftell(fin);
    if (cur >= 0 && fseek(fin, 0, SEEK_END) == 0) {
        const long end = ftell(fin);
        if (end >= cur) words = (end - cur) / 4;
    }
    if (words < 0) {                         /* not seekable: count as the reference does */
        unsigned int w;
        words = 0;
        while (fread(&w, sizeof(w), 1, fin) == 1) words++;
    }
    fseek(fin, 0, SEEK_SET);
    ktm_io_ok();
    return (int)words;
}

/* n words from the current position into a new malloc'd buffer, then back to
 * the start (ioFunctions.c:60-67, :69-76).  Where the file holds fewer than n,
 * the rest of the buffer is zero (the reference leaves it uninitialised) and
 * the status is KTM_ERR_IO. */
static void* read_n_words(FILE* fin, int n, const char* who)
{
    const size_t count = n > 0 ? (size_t)n : 0;
    unsigned char* p = (unsigned char*)calloc(count ? count : 1, 4);
    if (!p) {
        io_fail(KTM_ERR_NOMEM, "%s: cannot allocate %d words", who, n);
        return NULL;
    }
    if (!fin) {
        io_fail(KTM_ERR_ARG, "%s: NULL file", who);
        return p;
    }
    const size_t got = count ? fread(p, 4, count, fin) : 0;
    fseek(fin, 0, SEEK_SET);
    if (got < count) io_fail(KTM_ERR_IO, "%s: %zu of %d words read", who, got, n);
    else ktm_io_ok();
    return p;
}

unsigned int* binReadUints(FILE* fin, int n)
{
    return (unsigned int*)read_n_words(fin, n, "binReadUints");
}

float* binReadFloats(FILE* fin, int n)
{
    return (float*)read_n_words(fin, n, "binReadFloats");
}

/* t floats to fout (ioFunctions.c:79-83). */
void fileWrite(FILE* fout, float* ptr, int t)
{
    if (!fout || (t > 0 && !ptr)) {
        io_fail(KTM_ERR_ARG, "fileWrite: NULL file or buffer");
        return;
    }
    if (t > 0 && fwrite(ptr, sizeof(float), (size_t)t, fout) != (size_t)t) {
        io_fail(KTM_ERR_IO, "fileWrite: short write");
        return;
    }
    ktm_io_ok();
}

/* ioFunctions.c:87-90 */
void errorMessage(char* str)
{
    printf("Can't open %s.\n", str);
}

/* ioFunctions.c:94-153: the five input files of ../data (relative to the working
 * directory), opened "r+b" as the reference opens them; a file that cannot be
 * opened is reported on stdout (errorMessage) and sets flag = 1, the others are
 * still opened.  The status is KTM_ERR_IO when flag is set. */
void loadInputData(struct fileInputPtrs* input)
{
    static const char* const names[5] = {"../data/inputData.bin", "../data/inputSrcX.bin",
                                         "../data/inputSrcY.bin", "../data/inputRecX.bin",
                                         "../data/inputRecY.bin"};
    if (!input) {
        io_fail(KTM_ERR_ARG, "loadInputData: NULL input");
        return;
    }
    FILE** slot[5] = {&input->inputData, &input->inputSrcX, &input->inputSrcY,
                      &input->inputRecX, &input->inputRecY};
    input->flag = 0;
    for (int i = 0; i < 5; i++) {
        FILE* f = fopen(names[i], "r+b");
        if (!f) {
            errorMessage((char*)names[i]);
            input->flag = 1;
        } else {
            *slot[i] = f;
        }
    }
    if (input->flag) io_fail(KTM_ERR_IO, "loadInputData: an input file of ../data cannot be opened");
    else ktm_io_ok();
}
