/*
 * shwfs_setup.h -- host-side setup producers of the B200 Shack-Hartmann frame.
 *
 * When the frame runs inside the reference simulator, these arrays come from
 * its own setup (maos/powfs.c) and are passed through shwfs_b200.h.  A
 * standalone user builds them here instead.  Every producer restates the
 * reference routine cited beside it; geometry, valid-subaperture selection and
 * pixel-sampling maps are bit-for-bit the reference's.
 *
 * The matched filter is built as the reference builds it: i0 and its
 * derivatives from the short-exposure OTF of the turbulence and the uplink
 * (genseotf/genotf with piston, tip and tilt removed, lib/gensei.c:41-111,
 * lib/genotf.c:46-330; gensepsf, lib/gensei.c:135-209) times the ETF or the
 * DTF nominal (gensei, :213-419), then inverted as lib/mtch.c does.
 */
#ifndef SHWFS_SETUP_H
#define SHWFS_SETUP_H
#include <stdint.h>
#include "shwfs_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct shwfs_setup_cfg {
	double D, Din;      /* telescope diameter and central obstruction */
	int amp_binary;     /* 1: binary annulus sampled at the OPD points; 0: area-weighted (loc_circle_add) */
	int order;          /* subapertures across */
	double dsa, dx;     /* subaperture size, OPD sampling */
	double saat;        /* area threshold */
	int embfac, notf;   /* embedding factor; OTF size (0 = automatic) */
	int pixpsa;         /* pixels per side */
	double pixtheta;    /* pixel size (rad) */
	double pixblur;     /* pixel blur (fraction of a pixel) */
	double wvl;         /* wavelength */
	double hs;          /* guide star range (INFINITY for NGS) */
	double siglev;      /* photons per subaperture per frame */
	double rne, bkgrnd, bkgrndc;
	int gradtype;       /* SHWFS_GRAD_MF or SHWFS_GRAD_COG */
	int sigmatch, mtchcr;
	double cogthres, cogoff;
	int has_llt;
	double llt_d, llt_widthp, llt_ox, llt_oy;
	int na_n;           /* evenly sampled sodium profile */
	const double* na_h;
	const double* na_p;
	double r0, L0;      /* powfs.r0 (at 0.5 um) and powfs.L0 of the matched filter's short-exposure OTF;
	                       r0 <= 0 or infinite: no turbulence (diffraction-limited) */
} shwfs_setup_cfg;

typedef struct shwfs_setup shwfs_setup;

/* Runs the setup (geometry, DTF, pixel map, ETF, LLT, matched filter). */
int shwfs_setup_create(shwfs_setup** ps, const shwfs_setup_cfg* cfg);
void shwfs_setup_destroy(shwfs_setup* s);
const char* shwfs_setup_error(const shwfs_setup* s);

/* Scalars */
int shwfs_setup_nsa(const shwfs_setup* s);
int shwfs_setup_nopd(const shwfs_setup* s);
int shwfs_setup_notf(const shwfs_setup* s);
int shwfs_setup_npix(const shwfs_setup* s);
int shwfs_setup_llt_nx(const shwfs_setup* s);
double shwfs_setup_dx(const shwfs_setup* s);
double shwfs_setup_areascale(const shwfs_setup* s);
double shwfs_setup_dtheta(const shwfs_setup* s);
double shwfs_setup_i0sumsum(const shwfs_setup* s);
/* powfs.saasum as the reference forms it (maos/powfs.c:227-230). */
double shwfs_setup_saasum(const shwfs_setup* s);

/* Array getters (sizes in brackets); return SHWFS_EINVAL if the array does not exist. */
#define SHWFS_SETUP_SALOCX 1  /* [nsa] subaperture lower-left corner x */
#define SHWFS_SETUP_SALOCY 2  /* [nsa] */
#define SHWFS_SETUP_ORIGX 3   /* [nsa] first OPD point x */
#define SHWFS_SETUP_ORIGY 4   /* [nsa] */
#define SHWFS_SETUP_AMP 5     /* [nsa*nopd^2] */
#define SHWFS_SETUP_SAA 6     /* [nsa] */
#define SHWFS_SETUP_NOMINAL 7 /* [notf^2] treated DTF nominal */
#define SHWFS_SETUP_SIMAP_WT 8 /* [npix*4] */
#define SHWFS_SETUP_SROT 9    /* [nsa] */
#define SHWFS_SETUP_SRSA 10   /* [nsa] */
#define SHWFS_SETUP_ETF 11    /* [2*nsa*notf^2] interleaved complex, nominal fused */
#define SHWFS_SETUP_LLTAMP 12 /* [llt_nx^2] */
#define SHWFS_SETUP_MTCHE 13  /* [nsa*2*npix] */
#define SHWFS_SETUP_I0SUM 14  /* [nsa] */
#define SHWFS_SETUP_I0 15     /* [nsa*npix] */
#define SHWFS_SETUP_GX 16     /* [nsa*npix] */
#define SHWFS_SETUP_GY 17     /* [nsa*npix] */
#define SHWFS_SETUP_SEPSF 18  /* [nsa*notf^2] short-exposure PSF, peak in the centre (intstat.sepsf) */
#define SHWFS_SETUP_SEOTF 19  /* [2*nsa*notf^2] its OTF, peak in the corner, interleaved complex */
int shwfs_setup_get(const shwfs_setup* s, int what, double* out);
/* [npix*4] pixel-map tap indices into the notf^2 PSF, -1 for unused */
int shwfs_setup_get_simap_idx(const shwfs_setup* s, int* out);

/* Declares the powfs in a context and uploads every array; *ipowfs receives
   its index.  WFS are added separately (shwfs_wfs_add); the matched filter of
   the setup is available for shwfs_wfs_set_mtche via shwfs_setup_get. */
int shwfs_setup_load(const shwfs_setup* s, shwfs_ctx* ctx, int* ipowfs);
/* Declares the setup as another wavelength band of powfs ipowfs
   (shwfs_powfs_add_band, weight wvlwt) and uploads its pixel map and its ETF
   or DTF nominal; *iband receives the band's powfs index.  The setup is that
   of the same powfs configuration at the band's wavelength. */
int shwfs_setup_load_band(const shwfs_setup* s, shwfs_ctx* ctx, int ipowfs, double wvlwt, int* iband);
/* Loads the setup's matched filter (or CoG i0sum) into WFS iwfs. */
int shwfs_setup_load_wfs(const shwfs_setup* s, shwfs_ctx* ctx, int iwfs);

/* Von Karman phase screens as the reference generates them
   (lib/turbulence.c:70-168, spatial_psd :436-478): screens are made in
   pairs from one complex FFT; r0 at 0.5 um; wt[i] scales layer i's power.
   out[i] receives nx*ny values (x fastest). */
int shwfs_screens_vonkarman(double* const* out, int nlayer, long nx, long ny, double dx, double r0, double L0,
	const double* wt, uint32_t seed);

/* Science aperture of an annulus (D, Din) sampled at dx, as setup_aper
   builds it without loaded locs, amplitude map or pupil mask
   (maos/aper.c:45-110): create_metapupil with one guard point and
   loc_from_map (math/map.c:131-239, math/loc.c:448-492), mkamp's
   area-weighted annulus (loc_circle_add, math/loc.c:942-986), loc_reduce of
   each row's leading and trailing points below EPS (math/loc.c:1048-1128)
   and the amplitude normalised to sum 1.  With locx == NULL only *nloc is
   set; otherwise locx, locy, amp receive *nloc values (row by row, x
   fastest). */
int shwfs_aper_build(double D, double Din, double dx, long* nloc, double* locx, double* locy, double* amp);

#ifdef __cplusplus
}
#endif
#endif
