/*
 * ref_shim.h -- force-included when compiling the reference's own C sources
 * (src/psktmCPU.c, src/psktmFunctions.c, src/ioFunctions.c) into
 * oracle/_ref/libktm_ref.so.  The reference ships no headers: it uses
 * struct imageGrid / struct jobParams / struct fileInputPtrs, malloc and the
 * IBM masks without defining them.  This supplies them; the sources themselves
 * are compiled unmodified where they lie.  TEST INFRASTRUCTURE ONLY.
 */
#include <stdio.h>
#include <stdlib.h>
#include "../include/ktm.h"

/* IBM-32 field masks used by ioFunctions.c:22-29: bit 31 sign, bits 30-24
 * base-16 exponent, bits 23-0 fraction. */
#define SIGN_MASK 0x80000000u
#define EXPONENT_MASK 0x7f000000u
#define FRACTION_MASK 0x00ffffffu

/* struct fileInputPtrs (ioFunctions.c:96-148) comes from ktm.h, so that the
 * reference's loadInputData and the library's fill the same layout. */
