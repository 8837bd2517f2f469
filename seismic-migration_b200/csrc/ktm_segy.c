/*
 * ktm_segy.c -- SEG-Y (rev 0 layout) reader, the C replacement of the Octave
 * front end ktmGetInputMeta.m (:21-150) and ktmGetInputTrace.m (:29-75).
 *
 *   bytes 0..3199      textual reel header, 40 x 80 EBCDIC characters
 *   bytes 3200..3599   binary reel header: three 32-bit words (job, line, reel
 *                      numbers) then 16-bit words; the sample interval [us] at
 *                      3216, samples per trace at 3220, sample format at 3224
 *   then per trace     a 240-byte header and the samples (4 bytes for formats
 *                      1 IBM float, 2 int32, 5 IEEE float; 2 bytes for format
 *                      3 int16; 1 byte for format 8 int8)
 *
 * Fields are big-endian (the standard); bigEndian = 0 reads byte-swapped files
 * (the scripts' 'ieee-le' option).  Trace-header fields are decoded as signed
 * two's-complement values, so negative coordinates and scalars survive.
 * Samples come back as 4-byte words ready for ktm_job: IBM words unconverted
 * (KTM_FMT_IBM32, decoded on the GPU), every other format as float
 * (KTM_FMT_F32).
 */
#define _FILE_OFFSET_BITS 64
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>

#include "../../include/ktm.h"

int ktm_io_error(int code, const char* msg);
int ktm_io_ok(void);

static int segy_fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return ktm_io_error(code, buf);
}

/* EBCDIC -> ASCII for the characters ktmGetInputMeta.m:30-45 maps (letters,
 * digits, space and - / : # @ { } \ ~); every other byte becomes '?'. */
static void ebcdic_table(unsigned char t[256])
{
    memset(t, '?', 256);
    for (int i = 0; i < 9; i++) {
        t[0x81 + i] = (unsigned char)('a' + i);
        t[0x91 + i] = (unsigned char)('j' + i);
        t[0xC1 + i] = (unsigned char)('A' + i);
        t[0xD1 + i] = (unsigned char)('J' + i);
    }
    for (int i = 0; i < 8; i++) {
        t[0xA2 + i] = (unsigned char)('s' + i);
        t[0xE2 + i] = (unsigned char)('S' + i);
    }
    for (int i = 0; i < 10; i++) t[0xF0 + i] = (unsigned char)('0' + i);
    t[0x40] = ' ';
    t[0x60] = '-';
    t[0x61] = '/';
    t[0x7A] = ':';
    t[0x7B] = '#';
    t[0x7C] = '@';
    t[0xA1] = '~';
    t[0xC0] = '{';
    t[0xD0] = '}';
    t[0xE0] = '\\';
    t[0xE1] = ' ';   /* the script maps it to NUL; a space keeps the text a C string */
}

static uint32_t get_u32(const unsigned char* p, int be)
{
    return be ? ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]
              : ((uint32_t)p[3] << 24) | ((uint32_t)p[2] << 16) | ((uint32_t)p[1] << 8) | p[0];
}

static uint16_t get_u16(const unsigned char* p, int be)
{
    return be ? (uint16_t)(((unsigned)p[0] << 8) | p[1]) : (uint16_t)(((unsigned)p[1] << 8) | p[0]);
}

static int sample_bytes(int format)
{
    switch (format) {
        case 1: case 2: case 5: return 4;
        case 3: return 2;
        case 8: return 1;
        default: return 0;
    }
}

int ktmSegyOpen(const char* path, int bigEndian, ktm_segy_info* info)
{
    if (!path || !info) return segy_fail(KTM_ERR_ARG, "NULL argument");
    memset(info, 0, sizeof(*info));
    FILE* f = fopen(path, "rb");
    if (!f) return segy_fail(KTM_ERR_IO, "cannot open %s", path);
    unsigned char head[3600];
    size_t got = fread(head, 1, sizeof(head), f);
    long long size = -1;
    if (fseeko(f, 0, SEEK_END) == 0) size = (long long)ftello(f);
    fclose(f);
    if (got != sizeof(head) || size < 3600)
        return segy_fail(KTM_ERR_IO, "%s: shorter than the 3600-byte reel headers", path);
    const int be = bigEndian != 0;
    unsigned char tbl[256];
    ebcdic_table(tbl);
    for (int r = 0; r < 40; r++) {
        for (int c = 0; c < 80; c++) info->text[r * 81 + c] = (char)tbl[head[r * 80 + c]];
        info->text[r * 81 + 80] = '\n';
    }
    info->text[40 * 81 - 1] = '\0';
    const unsigned char* b = head + 3200;
    for (int i = 0; i < 3; i++) info->reel32[i] = get_u32(b + 4 * i, be);
    for (int i = 0; i < 24; i++) info->reel16[i] = get_u16(b + 12 + 2 * i, be);
    info->sampleInterval = info->reel16[2];       /* bytes 3217-3218 */
    info->samplesPerTrace = info->reel16[4];      /* bytes 3221-3222 */
    info->format = info->reel16[6];               /* bytes 3225-3226 */
    info->bigEndian = be;
    const int sb = sample_bytes(info->format);
    if (!sb)
        return segy_fail(KTM_ERR_IO, "%s: sample format %d (1 IBM, 2 int32, 3 int16, 5 IEEE, 8 int8 "
                                     "are read)", path, info->format);
    if (info->samplesPerTrace <= 0)
        return segy_fail(KTM_ERR_IO, "%s: %d samples per trace", path, info->samplesPerTrace);
    info->traceBytes = 240 + (long long)sb * info->samplesPerTrace;
    info->traceCount = (size - 3600) / info->traceBytes;
    return ktm_io_ok();
}

/* one 240-byte trace header, grouped as ktmGetInputMeta.m:132 returns it:
 * 7 x int32 (bytes 1-28), 4 x int16 (29-36), 8 x int32 (37-68), 2 x int16 (69-72),
 * 4 x int32 (73-88), 76 x int16 (89-240) */
static void decode_header(const unsigned char* h, int be, ktm_segy_trace* t)
{
    int k = 0;
    for (int i = 0; i < 7; i++) t->values[k++] = (int32_t)get_u32(h + 4 * i, be);
    for (int i = 0; i < 4; i++) t->values[k++] = (int16_t)get_u16(h + 28 + 2 * i, be);
    for (int i = 0; i < 8; i++) t->values[k++] = (int32_t)get_u32(h + 36 + 4 * i, be);
    for (int i = 0; i < 2; i++) t->values[k++] = (int16_t)get_u16(h + 68 + 2 * i, be);
    for (int i = 0; i < 4; i++) t->values[k++] = (int32_t)get_u32(h + 72 + 4 * i, be);
    for (int i = 0; i < 76; i++) t->values[k++] = (int16_t)get_u16(h + 88 + 2 * i, be);
    /* coordinate scalar (bytes 71-72): > 0 multiplier, < 0 divisor, 0 = 1 */
    const int sc = t->values[20];
    double* xy[4] = {&t->srcX, &t->srcY, &t->recX, &t->recY};
    for (int i = 0; i < 4; i++) {
        const double v = (double)t->values[21 + i];
        *xy[i] = sc > 0 ? v * (double)sc : (sc < 0 ? v / (double)(-sc) : v);
    }
}

int ktmSegyReadTraces(const char* path, const ktm_segy_info* info, long long first, long long count,
                      void* samples, ktm_segy_trace* headers)
{
    if (!path || !info) return segy_fail(KTM_ERR_ARG, "NULL argument");
    if (first < 0 || count < 0 || first + count > info->traceCount)
        return segy_fail(KTM_ERR_ARG, "traces [%lld, %lld) outside the file's %lld", first,
                         first + count, info->traceCount);
    if (count > 0 && !samples && !headers) return segy_fail(KTM_ERR_ARG, "nothing to read into");
    const int sb = sample_bytes(info->format);
    if (!sb || info->traceBytes != 240 + (long long)sb * info->samplesPerTrace)
        return segy_fail(KTM_ERR_ARG, "info does not come from ktmSegyOpen");
    FILE* f = fopen(path, "rb");
    if (!f) return segy_fail(KTM_ERR_IO, "cannot open %s", path);
    if (fseeko(f, (off_t)(3600 + first * info->traceBytes), SEEK_SET) != 0) {
        fclose(f);
        return segy_fail(KTM_ERR_IO, "%s: seek failed", path);
    }
    unsigned char* rec = (unsigned char*)malloc((size_t)info->traceBytes);
    if (!rec) {
        fclose(f);
        return segy_fail(KTM_ERR_NOMEM, "out of host memory");
    }
    const int be = info->bigEndian;
    const int ns = info->samplesPerTrace;
    int rc = KTM_OK;
    for (long long k = 0; k < count; k++) {
        if (fread(rec, 1, (size_t)info->traceBytes, f) != (size_t)info->traceBytes) {
            rc = segy_fail(KTM_ERR_IO, "%s: short read at trace %lld", path, first + k);
            break;
        }
        if (headers) decode_header(rec, be, headers + k);
        if (!samples) continue;
        const unsigned char* s = rec + 240;
        uint32_t* w = (uint32_t*)samples + (size_t)k * ns;
        float* x = (float*)samples + (size_t)k * ns;
        for (int j = 0; j < ns; j++) {
            switch (info->format) {
                case 1: w[j] = get_u32(s + 4 * j, be); break;           /* IBM word, decoded on the GPU */
                case 5: w[j] = get_u32(s + 4 * j, be); break;           /* IEEE bits */
                case 2: x[j] = (float)(int32_t)get_u32(s + 4 * j, be); break;
                case 3: x[j] = (float)(int16_t)get_u16(s + 2 * j, be); break;
                default: x[j] = (float)(int8_t)s[j]; break;
            }
        }
    }
    free(rec);
    fclose(f);
    return rc ? rc : ktm_io_ok();
}

int ktmSegyTraceFormat(const ktm_segy_info* info)
{
    return info && info->format == 1 ? KTM_FMT_IBM32 : KTM_FMT_F32;
}

int ktmLoadSegySurvey(const char* path, int bigEndian, long long first, long long count, int rebase,
                      ktm_survey* out)
{
    if (!path || !out) return segy_fail(KTM_ERR_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    ktm_segy_info info;
    int rc = ktmSegyOpen(path, bigEndian, &info);
    if (rc) return rc;
    if (count < 0) count = info.traceCount - first;
    if (first < 0 || count < 0 || first + count > info.traceCount)
        return segy_fail(KTM_ERR_ARG, "traces [%lld, %lld) outside the file's %lld", first,
                         first + count, info.traceCount);
    if (count > 0x7fffffffLL) return segy_fail(KTM_ERR_LIMIT, "too many traces");
    const size_t ntr = (size_t)count, nt = (size_t)info.samplesPerTrace;
    void* data = malloc(ntr * nt * 4 + 4);
    ktm_segy_trace* hdr = (ktm_segy_trace*)malloc(ntr * sizeof(ktm_segy_trace) + 1);
    out->midX = (float*)malloc(ntr * 4 + 4);
    out->midY = (float*)malloc(ntr * 4 + 4);
    out->offX = (float*)malloc(ntr * 4 + 4);
    out->offY = (float*)malloc(ntr * 4 + 4);
    if (!data || !hdr || !out->midX || !out->midY || !out->offX || !out->offY) {
        free(data); free(hdr);
        ktmFreeSurvey(out);
        return segy_fail(KTM_ERR_NOMEM, "out of host memory");
    }
    rc = ktmSegyReadTraces(path, &info, first, count, data, hdr);
    if (rc) {
        free(data); free(hdr);
        ktmFreeSurvey(out);
        return rc;
    }
    out->traces = data;
    out->traceFormat = ktmSegyTraceFormat(&info);
    out->inp.tracePts = info.samplesPerTrace;
    out->inp.sampleRate = (float)(info.sampleInterval * 1e-6);
    out->inp.traceNo = (int)count;
    double ox = 0.0, oy = 0.0;
    if (rebase && ntr > 0) {
        ox = fmin(hdr[0].srcX, hdr[0].recX);
        oy = fmin(hdr[0].srcY, hdr[0].recY);
        for (size_t k = 0; k < ntr; k++) {
            ox = fmin(ox, fmin(hdr[k].srcX, hdr[k].recX));
            oy = fmin(oy, fmin(hdr[k].srcY, hdr[k].recY));
        }
        ox = floor(ox);
        oy = floor(oy);
    }
    out->originX = ox;
    out->originY = oy;
    /* ktmConvertXYtoOffMid.m:12 in FP64 on the scaled coordinates */
    for (size_t k = 0; k < ntr; k++) {
        out->midX[k] = (float)((hdr[k].recX + hdr[k].srcX) / 2.0 - ox);
        out->midY[k] = (float)((hdr[k].recY + hdr[k].srcY) / 2.0 - oy);
        out->offX[k] = (float)((hdr[k].recX - hdr[k].srcX) / 2.0);
        out->offY[k] = (float)((hdr[k].recY - hdr[k].srcY) / 2.0);
    }
    free(hdr);
    return ktm_io_ok();
}
