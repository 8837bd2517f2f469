/*
 * ktm_oracle.h -- CPU oracle for the PSTM hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this code, and only as the checker.  The product (libktm.so) never
 * calls it.
 *
 * Two restatements of the reference algorithm live here:
 *   - oracle_migrate_ref32: psktmCPU.c:13-101 restated in single-threaded C,
 *     same float operations in the same order, so it is bit-identical to the
 *     reference run with one OpenMP thread.  Pinned by the golden fixtures in
 *     tests/golden/ that the reference's own code produced.
 *   - oracle_migrate_f64 / oracle_demigrate_f64 / oracle_vrms_grad_f64: the same
 *     method in FP64, extended with the features the fast kernels add and the reference lacks
 *     (linear trace interpolation, aperture, laterally varying Vrms cube).  With
 *     pick = truncate, no aperture and a 1-D velocity it is psktmCPU.c in FP64.
 */
#ifndef KTM_ORACLE_H
#define KTM_ORACLE_H

#include "../include/ktm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* axis[i] = start + (float)i * step  (psktmFunctions.c:1-39) */
void oracle_axis_f32(const struct imageGrid* g, float* axis);

/* psktmCPU.c:13-101, one thread, bit-identical. */
void oracle_migrate_ref32(const struct imageGrid* imageX, const struct imageGrid* imageY,
                          const struct imageGrid* imageZ, const struct jobParams* config,
                          const float* midX, const float* midY, const float* offX,
                          const float* offY, const float* traces, const float* slowness,
                          float* image);

/* FP64 description of one migration job (inputs are the float arrays the
 * library consumes; every operation is carried out in double). */
typedef struct oracle_job {
    struct imageGrid imageX, imageY, imageZ;
    int traceNo, tracePts, traceStride;
    double sampleRate;              /* trace sample interval, s */
    const float* midX; const float* midY; const float* offX; const float* offY;
    const float* traces;            /* [traceNo][traceStride] */
    const float* traceScale;        /* NULL or [traceNo] multiplier */
    const float* velocity;          /* [Nz] or [Nx][Ny][Nz] */
    int velocityCube;
    int pick;                       /* 0 truncate, 1 linear */
    double aperture;                /* <= 0: off */
    int prefold;                    /* 0: weight |tau| sqrt(t) per pair (psktmCPU.c:85);
                                       1: |tau| per pair and sqrt(j*dt) per trace sample,
                                          then interpolated; 2: as 1 but the samples
                                          given already carry sqrt(j*dt);
                                       3: |tau| times sqrt(j*dt) interpolated linearly
                                          at t/dt (the fast kernel's weight table) */
} oracle_job;

/* image[p] = sum_k w(p,k) * pick(trace_k, t(p,k)/dt); image overwritten.
 * Columns restricted to [col0, col0+ncol) of the Nx*Ny column list when ncol>0
 * (image then holds ncol*Nz values). */
void oracle_migrate_f64(const oracle_job* job, double* image, int col0, int ncol);

/* Exact transpose of oracle_migrate_f64 in linear or truncate mode:
 * data[k][j] = sum_p w(p,k) * coef_j(t(p,k)/dt) * image[p]; data overwritten
 * ([traceNo][traceStride]). */
void oracle_demigrate_f64(const oracle_job* job, const double* image, double* data);

/* dI[p]/dv[p]: derivative of each image sample with respect to the velocity at
 * that image sample (velocity cube semantics), linear pick. */
void oracle_vrms_grad_f64(const oracle_job* job, double* grad);

/* Count of (image point, trace) pairs inside the aperture (all pairs when off). */
unsigned long long oracle_count_aperture_pairs(const oracle_job* job);

/* ioFunctions.c:4-40 with SIGN_MASK 0x80000000, EXPONENT_MASK 0x7f000000,
 * FRACTION_MASK 0x00ffffff. */
void oracle_ibm32_to_ieee(const unsigned int* input, float* output, int n);

#ifdef __cplusplus
}
#endif
#endif
