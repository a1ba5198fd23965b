/*
 * Oracle-side initial conditions that the reference does not ship (test
 * infrastructure only; never linked into the product).
 *
 * The reference picks its initial data through cell_init_ptr /
 * cell_single_init_ptr (src/Cell/cell_init_function_ptr.c:6-46) over the enum
 * SHEAR..MIDDLE (src/Headers/header.h:8).  The oracle build compiles every
 * other reference source unchanged and replaces that one selector file with
 * ref_newic.c, which returns the reference's own routines for 0..6 and adds:
 *
 *   7  GRESHO        steady Gresho vortex (axisymmetric)
 *   8  KEPLER_RING   viscous Keplerian ring around a single point mass
 *   9  CIRCUMBINARY  r^-1/2 disk with an inner cavity around a binary
 *
 * Their extra parameters come from parfile keys that the reference reader
 * never asks for (so reference parfiles stay valid): IC_HoR, IC_Noise and
 * IC_Seed.  The driver reads them and stores them here before the first call.
 */
#ifndef ORACLE_REF_NEWIC_H
#define ORACLE_REF_NEWIC_H

enum { IC_GRESHO = 7, IC_KEPLER_RING = 8, IC_CIRCUMBINARY = 9 };

extern double oracle_ic_hor;   /* disk aspect ratio h/r (KEPLER_RING, CIRCUMBINARY) */
extern double oracle_ic_noise; /* relative amplitude of the seeded density noise */
extern int oracle_ic_seed;     /* seed of the density noise */

/* Uniform deviate in [-1, 1) for cell number idx of the reference's contiguous
 * (k, i, j) cell array: one splitmix64 step on (seed << 40) ^ idx, top 53 bits. */
double oracle_ic_noise_u(int seed, long idx);

#endif
