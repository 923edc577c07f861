/* CFD_diffusion.h -- drop-in for the reference's include/CFD_diffusion.h.
 * The reference's file holds 1D diffusion helpers that the Euler step never
 * calls; they are not part of the path this library provides, so this
 * header only exists for the reference's include list. */
#ifndef CFD_DIFFUSION_H
#define CFD_DIFFUSION_H
#endif
