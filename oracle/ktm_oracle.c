/*
 * ktm_oracle.c -- CPU oracle for the PSTM hot path.  TEST INFRASTRUCTURE ONLY:
 * loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker; never linked into or called by libktm.so.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off, no -march, so float
 * arithmetic is plain SSE with no FMA contraction, as in the reference build).
 *
 * Parity pin: oracle_migrate_ref32 is checked bit-for-bit against outputs of
 * the reference's own psktmCPU.c (tests/golden/, made by
 * tests/golden/make_golden.py from oracle/_ref/libktm_ref.so).
 */
#include "ktm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void oracle_axis_f32(const struct imageGrid* g, float* axis)
{
    /* psktmFunctions.c:26-33: start + (float)i * step, in float */
    for (int i = 0; i < g->imagePnts; i++) {
        float fi = (float)i;
        float prod = fi * g->imageStep;
        axis[i] = g->imageStart + prod;
    }
}

void oracle_migrate_ref32(const struct imageGrid* imageX, const struct imageGrid* imageY,
                          const struct imageGrid* imageZ, const struct jobParams* config,
                          const float* midX, const float* midY, const float* offX,
                          const float* offY, const float* traces, const float* slowness,
                          float* image)
{
    const int Li = imageX->imagePnts, Lj = imageY->imagePnts, Ll = imageZ->imagePnts;
    const float sRate = config->traceSampleRate;
    const int Nt = config->tracePts;

    float* xx = (float*)malloc(sizeof(float) * (size_t)(Li > 0 ? Li : 1));
    float* yy = (float*)malloc(sizeof(float) * (size_t)(Lj > 0 ? Lj : 1));
    float* zz = (float*)malloc(sizeof(float) * (size_t)(Ll > 0 ? Ll : 1));
    float* tau2 = (float*)malloc(sizeof(float) * (size_t)(Ll > 0 ? Ll : 1));
    float* slow2 = (float*)malloc(sizeof(float) * (size_t)(Ll > 0 ? Ll : 1));
    oracle_axis_f32(imageX, xx);
    oracle_axis_f32(imageY, yy);
    oracle_axis_f32(imageZ, zz);

    /* psktmCPU.c:46-49: tauS = ZZ^2, slownessS = 1/v^2 */
    for (int l = 0; l < Ll; l++) {
        tau2[l] = zz[l] * zz[l];
        float v2 = slowness[l] * slowness[l];
        slow2[l] = 1.0f / v2;
    }
    /* psktmCPU.c:52-53: image cleared, not accumulated into */
    memset(image, 0, sizeof(float) * (size_t)Li * (size_t)Lj * (size_t)Ll);

    /* psktmCPU.c:56-90: traces outermost, then x, y, tau; sums in trace order */
    for (int k = 0; k < config->traceNo; k++) {
        for (int i = 0; i < Li; i++) {
            /* :65-66 -- (mid - x - off)^2 and (mid - x + off)^2, evaluated left to right */
            float cs = (midX[k] - xx[i]) - offX[k];
            float cr = (midX[k] - xx[i]) + offX[k];
            float tC = cs * cs;
            float tD = cr * cr;
            for (int j = 0; j < Lj; j++) {
                /* :71-72 */
                float ds = (midY[k] - yy[j]) - offY[k];
                float dr = (midY[k] - yy[j]) + offY[k];
                float tA = tC + ds * ds;
                float tB = tD + dr * dr;
                float* col = image + ((size_t)i * Lj + j) * Ll;
                for (int l = 0; l < Ll; l++) {
                    /* :78-80 */
                    float t = sqrtf(tau2[l] + tA * slow2[l]);
                    t += sqrtf(tau2[l] + tB * slow2[l]);
                    int it = (int)(t / sRate);
                    /* :82-85 -- sample 0 and it >= tracePts excluded */
                    if (it < Nt && it > 0) {
                        float a = traces[it + (size_t)k * Nt] * t;
                        col[l] += a * sqrtf(tau2[l] / t);
                    }
                }
            }
        }
    }
    free(xx); free(yy); free(zz); free(tau2); free(slow2);
}

/* ---------------------------------------------------------------------- */
/* FP64 oracle of the extended method                                     */
/* ---------------------------------------------------------------------- */

static double axis_d(const struct imageGrid* g, int i)
{
    return (double)g->imageStart + (double)i * (double)g->imageStep;
}

static double vel_at(const oracle_job* job, int i, int j, int l)
{
    int Ny = job->imageY.imagePnts, Nz = job->imageZ.imagePnts;
    if (job->velocityCube)
        return (double)job->velocity[((size_t)i * Ny + j) * Nz + l];
    return (double)job->velocity[l];
}

static double sample_at(const oracle_job* job, int k, int j)
{
    /* reference sample window: 0 < j < tracePts (psktmCPU.c:82) */
    if (j <= 0 || j >= job->tracePts) return 0.0;
    double s = (double)job->traces[(size_t)k * job->traceStride + j];
    if (job->traceScale) s *= (double)job->traceScale[k];
    /* weight applied per sample: sqrt(t_j), t_j = j*dt */
    if (job->prefold == 1) s *= sqrt((double)j * job->sampleRate);
    return s;
}

/* Per-pair kinematics: returns 0 when the pair is outside the aperture. */
typedef struct pair_geo {
    double t, u, w;       /* traveltime (s), t/dt, weight */
    double as_, ar_;      /* tau^2 + D*S for each leg */
    double ds2, dr2;      /* squared horizontal distances */
} pair_geo;

static int pair_eval(const oracle_job* job, int k, double x, double y, double tau,
                     double v, pair_geo* g)
{
    double mx = job->midX[k], my = job->midY[k], ox = job->offX[k], oy = job->offY[k];
    if (job->aperture > 0.0) {
        double dmx = mx - x, dmy = my - y;
        if (dmx * dmx + dmy * dmy > job->aperture * job->aperture) return 0;
    }
    double sx = mx - ox - x, sy = my - oy - y, rx = mx + ox - x, ry = my + oy - y;
    g->ds2 = sx * sx + sy * sy;
    g->dr2 = rx * rx + ry * ry;
    double S = 1.0 / (v * v);
    double tau2 = tau * tau;
    g->as_ = tau2 + g->ds2 * S;
    g->ar_ = tau2 + g->dr2 * S;
    g->t = sqrt(g->as_) + sqrt(g->ar_);
    g->u = g->t / job->sampleRate;
    /* psktmCPU.c:85: w = t * sqrt(tau^2 / t)  (= |tau| sqrt(t)); with a per-sample
     * weight only the |tau| factor stays per pair */
    if (job->prefold == 3) {
        /* sqrt(t) by linear interpolation of sqrt(j*dt) between the samples around t */
        double fl = floor(g->u), f = g->u - fl;
        double dt = job->sampleRate;
        g->w = fabs(tau) * ((1.0 - f) * sqrt(fl * dt) + f * sqrt((fl + 1.0) * dt));
    } else if (job->prefold) {
        g->w = fabs(tau);
    } else {
        g->w = (g->t > 0.0) ? g->t * sqrt(tau2 / g->t) : 0.0;
    }
    return 1;
}

void oracle_migrate_f64(const oracle_job* job, double* image, int col0, int ncol)
{
    const int Nx = job->imageX.imagePnts, Ny = job->imageY.imagePnts;
    const int Nz = job->imageZ.imagePnts;
    int c0 = 0, c1 = Nx * Ny;
    if (ncol > 0) { c0 = col0; c1 = col0 + ncol; }
    for (int c = c0; c < c1; c++) {
        int i = c / Ny, j = c % Ny;
        double x = axis_d(&job->imageX, i), y = axis_d(&job->imageY, j);
        double* col = image + (size_t)(c - c0) * Nz;
        for (int l = 0; l < Nz; l++) col[l] = 0.0;
        for (int k = 0; k < job->traceNo; k++) {
            for (int l = 0; l < Nz; l++) {
                double tau = axis_d(&job->imageZ, l);
                pair_geo g;
                if (!pair_eval(job, k, x, y, tau, vel_at(job, i, j, l), &g)) break;
                double val;
                if (job->pick == 0) {
                    /* trunc toward zero; the index is only used inside 0 < it < Nt */
                    if (!(g.u < (double)job->tracePts)) continue;
                    int it = (int)g.u;
                    val = sample_at(job, k, it);
                } else {
                    if (!(g.u < (double)job->tracePts + 1.0)) continue;
                    double fl = floor(g.u);
                    int i0 = (int)fl;
                    double f = g.u - fl;
                    val = (1.0 - f) * sample_at(job, k, i0) + f * sample_at(job, k, i0 + 1);
                }
                col[l] += g.w * val;
            }
        }
    }
}

void oracle_demigrate_f64(const oracle_job* job, const double* image, double* data)
{
    const int Nx = job->imageX.imagePnts, Ny = job->imageY.imagePnts;
    const int Nz = job->imageZ.imagePnts, Nt = job->tracePts, st = job->traceStride;
    memset(data, 0, sizeof(double) * (size_t)job->traceNo * st);
    for (int k = 0; k < job->traceNo; k++) {
        double sc = job->traceScale ? (double)job->traceScale[k] : 1.0;
        double* d = data + (size_t)k * st;
        for (int c = 0; c < Nx * Ny; c++) {
            int i = c / Ny, j = c % Ny;
            double x = axis_d(&job->imageX, i), y = axis_d(&job->imageY, j);
            for (int l = 0; l < Nz; l++) {
                double tau = axis_d(&job->imageZ, l);
                pair_geo g;
                if (!pair_eval(job, k, x, y, tau, vel_at(job, i, j, l), &g)) break;
                double m = image[(size_t)c * Nz + l] * g.w * sc;
                if (job->pick == 0) {
                    if (!(g.u < (double)Nt)) continue;
                    int it = (int)g.u;
                    if (it > 0 && it < Nt) d[it] += m;
                } else {
                    if (!(g.u < (double)Nt + 1.0)) continue;
                    double fl = floor(g.u);
                    int i0 = (int)fl;
                    double f = g.u - fl;
                    if (i0 > 0 && i0 < Nt) d[i0] += (1.0 - f) * m;
                    if (i0 + 1 > 0 && i0 + 1 < Nt) d[i0 + 1] += f * m;
                }
            }
        }
        /* prefolded weight: the migration reads sample j times sqrt(j dt) (sample_at) */
        if (job->prefold == 1)
            for (int j = 1; j < Nt; j++) d[j] *= sqrt((double)j * job->sampleRate);
    }
}

void oracle_vrms_grad_f64(const oracle_job* job, double* grad)
{
    /* I[p] = sum_k w * val(u);  S = 1/v^2 at p;  dt/dS = D_s/(2 sqrt(a_s)) + D_r/(2 sqrt(a_r))
     * w = |tau| sqrt(t) (in-kernel weight) or |tau| (prefolded), val linear in u with
     * slope D(i0+1) - D(i0).  dI/dv = dI/dS * (-2 / v^3). */
    const int Nx = job->imageX.imagePnts, Ny = job->imageY.imagePnts;
    const int Nz = job->imageZ.imagePnts;
    for (int c = 0; c < Nx * Ny; c++) {
        int i = c / Ny, j = c % Ny;
        double x = axis_d(&job->imageX, i), y = axis_d(&job->imageY, j);
        for (int l = 0; l < Nz; l++) {
            double tau = axis_d(&job->imageZ, l);
            double v = vel_at(job, i, j, l);
            double acc = 0.0;
            for (int k = 0; k < job->traceNo; k++) {
                pair_geo g;
                if (!pair_eval(job, k, x, y, tau, v, &g)) continue;
                if (!(g.u < (double)job->tracePts + 1.0)) continue;
                if (g.as_ <= 0.0 || g.ar_ <= 0.0 || g.t <= 0.0) continue;
                double fl = floor(g.u);
                int i0 = (int)fl;
                double f = g.u - fl;
                double s0 = sample_at(job, k, i0), s1 = sample_at(job, k, i0 + 1);
                double val = (1.0 - f) * s0 + f * s1;
                double dval_du = s1 - s0;
                double dt_dS = g.ds2 / (2.0 * sqrt(g.as_)) + g.dr2 / (2.0 * sqrt(g.ar_));
                double dw_dt;
                if (job->prefold == 3)      /* table weight: slope of the interpolated sqrt(j dt) */
                    dw_dt = fabs(tau) * (sqrt((fl + 1.0) * job->sampleRate) - sqrt(fl * job->sampleRate)) / job->sampleRate;
                else
                    dw_dt = job->prefold ? 0.0 : fabs(tau) / (2.0 * sqrt(g.t));
                acc += (dw_dt * val + g.w * dval_du / job->sampleRate) * dt_dS;
            }
            grad[(size_t)c * Nz + l] = acc * (-2.0 / (v * v * v));
        }
    }
}

unsigned long long oracle_count_aperture_pairs(const oracle_job* job)
{
    const int Nx = job->imageX.imagePnts, Ny = job->imageY.imagePnts;
    unsigned long long n = 0;
    double a2 = job->aperture * job->aperture;
    for (int c = 0; c < Nx * Ny; c++) {
        int i = c / Ny, j = c % Ny;
        double x = axis_d(&job->imageX, i), y = axis_d(&job->imageY, j);
        for (int k = 0; k < job->traceNo; k++) {
            double dmx = job->midX[k] - x, dmy = job->midY[k] - y;
            if (job->aperture <= 0.0 || dmx * dmx + dmy * dmy <= a2) n++;
        }
    }
    return n * (unsigned long long)job->imageZ.imagePnts;
}

void oracle_ibm32_to_ieee(const unsigned int* input, float* output, int n)
{
    /* ioFunctions.c:18-38: sign * (fraction / FRACTION_MASK) * 16^(exponent - 64) */
    for (int i = 0; i < n; i++) {
        unsigned int w = input[i];
        float sign = (w & 0x80000000u) ? -1.0f : 1.0f;
        unsigned int fraction = w & 0x00ffffffu;
        float e = (float)(((w & 0x7f000000u) >> 24) & 127u) - 64.0f;
        float q = (float)fraction / (float)0x00ffffffu;
        output[i] = sign * q * powf(16.0f, e);
    }
}
