/*
 * shwfs_evl.h -- science-path evaluation on the B200: ray trace of the
 * turbulence onto the science aperture, wavefront-error statistics and the
 * time-averaged PSF, per science direction.
 *
 * It serves the open-loop part of the reference's performance evaluation
 * (gpu_perfevl_queue / gpu_perfevl_sync, cuda/sim/perfevl.cu:336-550;
 * perfevl_ievl, maos/perfevl.c:111-240): atm2loc onto aper->locs,
 * calc_ptt / loc_calc_ptt (math/loc.c:653-709) for the piston, tip/tilt and
 * piston-tip-tilt-removed variances and the mode coefficients, and
 * psfcomp_r / locfft_psf (lib/locfft.c:110-175) for the PSF: the wavefront
 * amp*exp(2*pi*i*OPD/wvl) embedded by loc_create_embed (math/loc.c:147-179)
 * in an nembed x nembed grid, forward FFT, |.|^2, corner-to-centre crop to
 * psfsize x psfsize (X(cpcorner2center), math/mat.c:745-767), accumulated
 * over frames.  Deformable mirrors, NCPA surfaces and closed-loop terms are
 * not part of this path.
 *
 * The aperture must be a regular grid of spacing dx (aper->locs is).  The
 * screens are those given to shwfs_atm_set; the frame index and dt are the
 * WFS path's.
 */
#ifndef SHWFS_EVL_H
#define SHWFS_EVL_H
#include "shwfs_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Science aperture (aper->locs and aper->amp, maos/aper.c:32-130): nloc
   points on a grid of spacing dx and their amplitude (the reference
   normalises it to sum 1).  The moment matrix of loc_mcc_ptt and its
   inverse (aper->mcc, ipcc, imcc) are formed here in FP64. */
int shwfs_evl_set_aper(shwfs_ctx* ctx, long nloc, const double* locx, const double* locy, double dx,
	const double* amp);
/* A science direction (parms->evl.thetax/thetay/hs; hs INFINITY for a
   star at infinity). */
int shwfs_evl_add_dir(shwfs_ctx* ctx, double thetax, double thetay, double hs, int* ievl);
/* PSF settings per wavelength (parms->evl.wvl, psfgridsize -> nembed,
   psfsize): nembed a power of two from 64 to 4096, psfsize even and at most
   nembed (0 = nembed).  pttr: remove piston/tip/tilt before the PSF
   (parms->evl.pttr), else the OPD is used as is.  Resets the PSF sums. */
int shwfs_evl_set_psf(shwfs_ctx* ctx, int nwvl, const double* wvl, const int* nembed, const int* psfsize, int pttr);
/* Queue the evaluation of frame isim for every direction on the context's
   stream: ray trace, WFE sums and, with do_psf, one PSF per wavelength
   added to the sums. */
int shwfs_evl_queue(shwfs_ctx* ctx, int isim, int do_psf);
/* Wait for the queued evaluation; per direction (nevl x 3, direction
   slowest): wfe = {PR, TT, PTTR} variances (m^2) and coeff = {piston, tip,
   tilt} as calc_ptt_post / loc_calc_ptt give them.  Either may be NULL. */
int shwfs_evl_sync(shwfs_ctx* ctx, double* wfe, double* coeff);
/* The accumulated PSF of direction ievl at wavelength iwvl (psfsize^2,
   column-major, centred) and the number of frames in it. */
int shwfs_evl_psf_get(shwfs_ctx* ctx, int ievl, int iwvl, double* psf, long* nframe);
/* Zero every PSF sum. */
int shwfs_evl_psf_reset(shwfs_ctx* ctx);
/* The OPD (nloc, aperture order) of direction ievl from the last queued
   frame, into a device buffer. */
int shwfs_evl_opd_dev(shwfs_ctx* ctx, int ievl, float* opd);

#ifdef __cplusplus
}
#endif
#endif
