/*
 * shwfs_b200.h -- C ABI of the B200 Shack-Hartmann wavefront-sensor frame.
 *
 * One frame of a physical-optics Shack-Hartmann WFS, per WFS:
 *   (a) ray trace of the turbulence layers into the subaperture OPD points,
 *   (b) field  amp*exp(i*2*pi*opd/wvl) embedded in an n_w x n_w grid,
 *   (c) |FFT|^2 -> PSF -> FFT -> OTF x uplink OTF* x (ETF or DTF nominal)
 *       -> inverse FFT -> real part sampled onto the detector pixels,
 *   (d) photon (Poisson) and read-out (Gaussian) noise,
 *   (e) centre-of-gravity or matched-filter gradients.
 *
 * The entry points replace the GPU seam of the reference simulator
 * (cuda/sim/gpu_sim.h:39-48): the static data that the reference uploads in
 * gpu_wfsgrad_init / gpu_wfsgrad_update_etf / gpu_wfsgrad_update_ref /
 * gpu_atm2gpu / gpu_wfsgrad_seeding is passed here as plain arrays, and
 * gpu_wfsgrad_queue + gpu_wfsgrad_sync become shwfs_frame_queue +
 * shwfs_frame_sync.  All arrays use the reference's layouts: column-major
 * (x fastest), subaperture-major, complex numbers as interleaved (re, im).
 * Angles are in radians, lengths in metres.
 *
 * Every call returns 0 on success or a negative SHWFS_E* code; the message of
 * the last failure on a context is returned by shwfs_last_error().  Calls on
 * one context must not overlap from several host threads; distinct contexts
 * are independent.
 */
#ifndef SHWFS_B200_H
#define SHWFS_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define SHWFS_OK 0
#define SHWFS_EINVAL (-1)   /* invalid argument or size */
#define SHWFS_ECUDA (-2)    /* CUDA runtime error */
#define SHWFS_ESTATE (-3)   /* call out of order (missing setup) */
#define SHWFS_ENOMEM (-4)   /* device allocation failed or over budget */
#define SHWFS_ETIMEOUT (-5) /* a bounded device wait expired */

typedef struct shwfs_ctx shwfs_ctx;

/* Gradient algorithms (maos/utils.c:983-1122, cuda/sim/wfsgrad.cu:413-478). */
#define SHWFS_GRAD_MF 1   /* matched filter, PTYPE_MF */
#define SHWFS_GRAD_COG 2  /* thresholded centre of gravity, PTYPE_COG */
#define SHWFS_GRAD_ZTILT 3 /* geometric: z-tilt of the OPD, no imaging (gtype_sim=GTYPE_Z) */
#define SHWFS_GRAD_GTILT 4 /* geometric: averaged gradient GS0*OPD, no imaging (gtype_sim=GTYPE_G) */

/* Imaging forms. */
#define SHWFS_FORM_FFT 0  /* FP32 shared-memory/register FFT */
#define SHWFS_FORM_TC 1   /* DFT as BF16x3 split products on tcgen05 tensor cores */

/*
 * Static description of one powfs (a group of identical WFS).  Mirrors the
 * fields of the reference's powfs_cfg_t / powfs_t that the frame reads
 * (maos/parms.h:152-330, maos/types.h powfs_t).
 */
typedef struct shwfs_powfs_desc {
	int nsa;          /* valid subapertures (powfs.saloc->nloc) */
	int nopd;         /* OPD points per subaperture side (pts->nxsa) */
	int embfac;       /* embedding factor, n_w = nopd*embfac */
	int notf;         /* OTF size n_f (powfs.notfx == notfy) */
	int pixpsax;      /* detector pixels along x */
	int pixpsay;      /* detector pixels along y */
	double pixthetax; /* pixel size along x (radpixtheta) */
	double pixthetay; /* pixel size along y (pixtheta) */
	double wvl;       /* wavelength (single band) */
	double dsa;       /* subaperture size (pts->dsa) */
	double dx;        /* OPD sampling (pts->dx) */
	double areascale; /* powfs.areascale */
	double hs;        /* guide star range; INFINITY for NGS */
	int has_etf;      /* 1: per-subaperture ETF with the nominal fused (LGS) */
	int has_llt;      /* 1: compute the uplink OTF from the LLT OPD each frame */
	int llt_nx;       /* LLT pupil points per side (llt->pts->nxsa) */
	double llt_ox, llt_oy; /* LLT position in the pupil */
	double llt_origx, llt_origy; /* llt->pts->origx[0], origy[0] */
	int gradtype;     /* SHWFS_GRAD_MF or SHWFS_GRAD_COG */
	int sigmatch;     /* 0, 1 or 2 (powfs.sigmatch) */
	double cogthres;  /* powfs.cogthres */
	double cogoff;    /* powfs.cogoff */
	double rne;       /* read noise per pixel (e-) */
	double bkgrnd;    /* background per pixel per frame (bkgrnd*dtrat) */
	double bkgrndc;   /* calibrated background per pixel per frame (bkgrnd*dtrat*bkgrndc) */
	double saat;      /* subaperture area threshold (CoG skips saa<saat) */
	double sigtot_cog;/* expected signal for sigmatch==0 CoG (siglev*dtrat) */
} shwfs_powfs_desc;

/* One WFS of a powfs (maos/parms.h wfs_cfg_t). */
typedef struct shwfs_wfs_desc {
	int ipowfs;
	double thetax, thetay; /* direction */
	double hs;             /* range of the star (INFINITY for NGS) */
	double hc;             /* conjugation height of the pupil (0) */
	double misregx, misregy;
	double sigsim;         /* photons per full subaperture per frame */
	double wvlwt;          /* wavelength weight (single band: 1) */
	int noisy;             /* add photon and read noise */
} shwfs_wfs_desc;

/* One turbulence layer (map_t with wind; cuda/sim/atm.cu). */
typedef struct shwfs_layer_desc {
	long nx, ny;      /* screen size (x fastest) */
	double dx;        /* screen sampling */
	double ox, oy;    /* coordinate of screen element (0,0) */
	double ht;        /* altitude */
	double vx, vy;    /* wind velocity */
	double alpha;     /* scaling (atmscale*wt) */
} shwfs_layer_desc;

/* ---- context ---- */
int shwfs_create(shwfs_ctx** pctx, int device);
int shwfs_destroy(shwfs_ctx* ctx);
const char* shwfs_last_error(const shwfs_ctx* ctx);
/* Version string of the library build. */
const char* shwfs_version(void);

/* ---- static data (replaces gpu_wfsgrad_init, cuda/sim/wfsinit.cu:159) ---- */
/* Declares a powfs; *ipowfs receives its index. */
int shwfs_powfs_add(shwfs_ctx* ctx, const shwfs_powfs_desc* desc, int* ipowfs);
/* Subaperture OPD-grid origins pts->origx/origy (nsa each) and the amplitude
   map powfs.amp (namp x nsa*nopd^2; namp is 1 or the number of WFS). */
int shwfs_powfs_set_geom(shwfs_ctx* ctx, int ipowfs, const double* origx, const double* origy,
	const double* amp, int namp, const double* saa);
/* DTF nominal (dtf[0].nominal, notf^2 real, treated: peak in corner with the
   fftshift folded in, lib/mkdtf.c:26-80); nnominal is 1 or nsa. */
int shwfs_powfs_set_nominal(shwfs_ctx* ctx, int ipowfs, const double* nominal, int nnominal);
/* Pixel sampling map (dtf[0].si, lib/mkdtf.c:158-161 via lib/mkh.c:62):
   for each of nmap maps (1 or nsa) and each pixel, up to 4 (index, weight)
   pairs into the notf^2 PSF; index -1 marks an unused slot.
   idx/wt: nmap*npix*4 entries. */
int shwfs_powfs_set_simap(shwfs_ctx* ctx, int ipowfs, const int* idx, const double* wt, int nmap);
/* Elongation transfer function with the nominal fused in
   (etfsim[0].etf, nsa x notf^2 complex; lib/mkdtf.c:186-396).
   slot 0 = etf[0]; slot 1 = second profile for time interpolation
   (gpu_wfsgrad_update_etf, cuda/sim/wfsinit.cu:32). */
int shwfs_powfs_set_etf(shwfs_ctx* ctx, int ipowfs, const double* etf, int slot);
/* LLT pupil amplitude (llt->amp, llt_nx^2). */
int shwfs_powfs_set_lltamp(shwfs_ctx* ctx, int ipowfs, const double* lltamp);
/* Short-exposure OTF of every subaperture (nsa x notf^2 complex, peak in the
   corner, x fastest), from which shwfs_wfs_update_mtche forms i0, gx and gy:
   the OTF of the p/t/t-removed turbulence (genseotf, lib/gensei.c:81-111)
   times the conjugate uplink OTF, to the PSF times saa/n^2 (intstat.sepsf,
   gensepsf :135-209), back to the OTF times 1/n^2 (gensei :327-335).
   shwfs_setup_load uploads the setup's (SHWFS_SETUP_SEOTF); NULL removes it,
   and update_mtche then uses the flat-wavefront OTF. */
int shwfs_powfs_set_seotf(shwfs_ctx* ctx, int ipowfs, const double* seotf);

/* Another wavelength band of powfs ipowfs (the reference images every
   wavelength of powfs.wvl, maos/wfsints.c:145-288; cuda/sim/wfsints.cu).  desc
   describes the band: the subapertures, sampling, sizes, pixels, LLT and
   gradient options of ipowfs, its own wvl; wvlwt is its weight
   (powfs.wvlwts[iwvl]); the main band's weight is the WFS's wvlwt.  *iband
   receives the band's powfs index: give the band its transfer functions and
   pixel map with shwfs_powfs_set_nominal / set_simap / set_etf (and
   set_lltamp to replace the LLT pupil copied from ipowfs).  The band copies
   the geometry of ipowfs as set at the call (set it first).  A frame of
   ipowfs's WFS traces the OPD once, images it in every band (the uplink OTF at
   each band's wavelength), sums the intensities, then adds noise and forms
   gradients once.  Matched filters come from the host for such a powfs
   (shwfs_wfs_update_mtche refuses it), and the work-list and allocation-free
   paths do not serve it; nor does shwfs_ints_grad_dev when ipowfs has an LGS
   uplink, whose per-band uplink OTFs only the frame path forms.  At most
   SHWFS_MAX_BANDS extra bands. */
#define SHWFS_MAX_BANDS 8
int shwfs_powfs_add_band(shwfs_ctx* ctx, int ipowfs, const shwfs_powfs_desc* desc, double wvlwt, int* iband);

/* Declares a WFS; *iwfs receives its index. */
int shwfs_wfs_add(shwfs_ctx* ctx, const shwfs_wfs_desc* desc, int* iwfs);
/* Matched filter mtche (nsa x 2 x npix, each subaperture a 2 x npix
   column-major block), i0sum (nsa) and i0sumsum (gpu_wfsgrad_update_ref,
   cuda/sim/wfsinit.cu:107). i0sum may be NULL for CoG. */
int shwfs_wfs_set_mtche(shwfs_ctx* ctx, int iwfs, const double* mtche, const double* i0sum, double i0sumsum);
/* The matched filter, i0 sums and their total held for WFS iwfs (set by
   shwfs_wfs_set_mtche or formed by shwfs_wfs_update_mtche), copied to host
   memory in the layout of shwfs_wfs_set_mtche; any pointer may be NULL.
   The reverse of gpu_wfsgrad_update_ref (cuda/sim/wfsinit.cu:107). */
int shwfs_wfs_get_mtche(shwfs_ctx* ctx, int iwfs, double* mtche, double* i0sum, double* i0sumsum);
/* The matched filter of WFS iwfs regenerated on the device from the powfs's
   short-exposure OTF (shwfs_powfs_set_seotf; else the OTF of a flat wavefront
   and flat uplink), current ETF (with its interpolation weights) or DTF
   nominal and pixel map, in place of a host-built one (the reference
   builds it on the host, lib/gensei.c:213-419 and lib/mtch.c:93-335, and
   copies it with gpu_wfsgrad_update_ref, cuda/sim/gpu_sim.h:42): i0 and its
   x/y derivatives of a flat wavefront, then the weighted pseudo-inverse with
   mtchcr's cross-coupling terms (0: none, 1: x and y, 2: x, 3: y), the
   eigenvalue thresholds of dpinv and the dim-subaperture and
   noise-equivalent-angle rejections.  i0sum and i0sumsum are set too.
   16x16 OPD points, FFT 32, one shared pixel map. */
int shwfs_wfs_update_mtche(shwfs_ctx* ctx, int iwfs, int mtchcr);
/* ETF time interpolation (maos/wfsints.c:215-223): with ETF slots 0 and 1
   set and dtrat > 0, frame isim uses ETF0 (1 - w) + ETF1 w with
   w = (isim mod dtrat) / dtrat; dtrat 0 uses slot 0 alone. */
int shwfs_powfs_set_etf_dtrat(shwfs_ctx* ctx, int ipowfs, int dtrat);
/* powfs.saasum (maos/powfs.c:227-230), the divisor of the CoG signal level
   under sigmatch 2 (maos/utils.c:1033-1035); shwfs_powfs_set_geom sets it to
   the sum of the saa it is given. */
int shwfs_powfs_set_saasum(shwfs_ctx* ctx, int ipowfs, double saasum);
/* Frames integrated per output frame (powfs.dtrat): the intensities of
   frames isim with isim mod dtrat = 0 .. dtrat-1 add up in each WFS's
   intensity buffer, and on the last one (isim + 1 a multiple of dtrat) the
   noise is drawn on the sum and the gradients are formed; other frames leave
   the gradients as they were.  1 (the default) forms every frame. */
int shwfs_powfs_set_dtrat(shwfs_ctx* ctx, int ipowfs, int dtrat);
/* Geometric (z-tilt) gradients (device, 2*nsa) of WFS iwfs from a device OPD
   (nsa*nopd^2): cuztilt (cuda/sim/wfsgrad.cu:57-106). */
int shwfs_grad_ztilt_dev(shwfs_ctx* ctx, int iwfs, const float* opd, float* grad);
/* Noise of geometric gradients (add_geom_noise_do, cuda/sim/wfsgrad.cu:39-51)
   for a noisy WFS of a geometric powfs: nea is 3*nsa, the lower Cholesky
   factor of each subaperture's NEA in radians (xx, yy, xy); null removes it. */
int shwfs_wfs_set_neasim(shwfs_ctx* ctx, int iwfs, const double* nea);
/* G-tilt operator of a geometric powfs (powfs.GS0, maos/powfs.c:607-632, made
   by mkg, lib/mkg.c:471): a MAOS sparse matrix (CSC, spint = int) of 2*nsa
   rows and nsa*nopd^2 columns; iamp selects the matrix of WFS wfsind = iamp
   when the powfs has one amplitude per WFS (else 0). */
int shwfs_powfs_set_gs0(shwfs_ctx* ctx, int ipowfs, int iamp, long nrow, long ncol, const int* pp,
	const int* pi, const double* px);
/* G-tilt gradients (device, 2*nsa) of WFS iwfs from a device OPD. */
int shwfs_grad_gtilt_dev(shwfs_ctx* ctx, int iwfs, const float* opd, float* grad);
/* Noise seed of one WFS (gpu_wfsgrad_seeding, cuda/sim/wfsinit.cu:532). */
int shwfs_wfs_seed(shwfs_ctx* ctx, int iwfs, uint64_t seed);

/* Turbulence screens (gpu_atm2gpu, cuda/sim/atm.cu:106): nlayer layers, FP64
   host screens converted to FP32 device screens (screens[i] has nx*ny). */
int shwfs_atm_set(shwfs_ctx* ctx, int nlayer, const shwfs_layer_desc* layers, const double* const* screens);

/* ---- closed loop and static surfaces (maos/wfsgrad.c:200-262,
        cuda/sim/wfsgrad.cu:531-605) ---- */
/* Deformable-mirror surfaces (gpu_dmreal2gpu, cuda/sim/atm.cu:315): ndm grids
   (x fastest, FP64 host values stored FP32) with their sampling, origin,
   conjugation height and weight alpha (-1 subtracts the mirror, as
   mapcell2loc(..., -1) does at cuda/sim/wfsgrad.cu:564-567; vx, vy are
   ignored).  A WFS that uses them (shwfs_wfs_set_opd_terms) traces them after
   the turbulence with its cone and misregistration, without wind and without
   wrap: a point whose bilinear cell leaves a grid gets nothing from it
   (map2loc_linear, cuda/sim/accphi.cu:24-38).  The first call allocates the
   grids; later calls with the same sizes only copy the new surfaces,
   asynchronously on the context stream (counted by shwfs_copy_counters), and
   apply to the frames queued after them.  ndm = 0 removes the mirrors.  The
   layers and mirrors together are at most 16. */
int shwfs_dm_set(shwfs_ctx* ctx, int ndm, const shwfs_layer_desc* dms, const double* const* surfaces);
/* Per-WFS terms of the OPD of the frames queued from now on (they persist
   until changed):
     use_dm     subtract the mirror grids of shwfs_dm_set (sim.closeloop);
     ptt        ptt[0] + ptt[1] x + ptt[2] y on the pupil points (loc_add_ptt,
                math/loc.c:762-789): -ttmreal and -fsmreal in closed loop,
                the telescope wind shake; NULL for none;
     focus_tel  f (x^2 + y^2) less its mean over the pupil points
                (loc_add_focus, math/loc.c:1247): -telfocusreal;
     focus_llt  the same about the LLT position llt_ox, llt_oy of the powfs
                descriptor (loc_add_focus_offset, math/loc.c:1226-1246):
                zoomfocusadj (maos/utils.c:865-879);
     lltptt     tip/tilt of the LLT pupil (wfsgrad_llt_tt,
                maos/wfsgrad.c:89-116, added at :373-377); NULL for none.
   LLT tip/tilt on a powfs without an LLT is refused. */
int shwfs_wfs_set_opd_terms(shwfs_ctx* ctx, int iwfs, int use_dm, const double* ptt, double focus_tel,
	double focus_llt, const double* lltptt);
/* Static surface added to WFS iwfs's OPD every frame (powfs.opdadd[wfsind],
   maos/wfsgrad.c:230-233; gpu_wfssurf2gpu, cuda/sim/wfsinit.cu:514-524):
   nsa*nopd^2 FP64 values on the pupil points, or NULL to remove it. */
int shwfs_wfs_set_opdadd(shwfs_ctx* ctx, int iwfs, const double* opd);

/* Imaging form used by the frame calls (default SHWFS_FORM_FFT). */
int shwfs_set_form(shwfs_ctx* ctx, int form);
/* Wind shift time step: frame isim shifts layer l by -v*dt*isim. */
int shwfs_set_dt(shwfs_ctx* ctx, double dt);

/* ---- per frame (replaces gpu_wfsgrad_queue / gpu_wfsgrad_sync) ---- */
/* Queue one frame of every WFS in [iwfs0, iwfs1) on the context stream:
   ray trace, imaging, noise, gradients.  Asynchronous. */
int shwfs_frame_queue(shwfs_ctx* ctx, int isim, int iwfs0, int iwfs1);
/* Wait for the queued frame and copy WFS iwfs's gradients (2*nsa: x then y)
   and optionally its pixel intensities (nsa*npix) to host memory. */
int shwfs_frame_sync(shwfs_ctx* ctx, int iwfs, double* grad, double* ints);
/* The frame of shwfs_frame_queue as one CUDA graph: the first call for a WFS
   range runs the frame normally (allocations, descriptor uploads, stream
   branches); later calls capture the frame's launches, update the
   instantiated graph with this frame's parameters and launch it.  The WFS of
   several powfs run as parallel branches of the graph.  Results are read
   with shwfs_frame_sync as after shwfs_frame_queue.  Stage profiling must be
   off.  Replaces the per-WFS gpu_wfsgrad_queue threads of
   cuda/sim/gpu_sim.h:45 for a whole frame. */
int shwfs_frame_graph(shwfs_ctx* ctx, int isim, int iwfs0, int iwfs1);
/* Gradients of WFS iwfs0..iwfs1-1 after their frame, one wait for all:
   grad (host) receives each WFS's 2*nsa values in turn.  The range form of
   shwfs_frame_sync for the gpu_wfsgrad_sync calls of one step
   (cuda/sim/gpu_sim.h:46). */
int shwfs_frame_sync_range(shwfs_ctx* ctx, int iwfs0, int iwfs1, double* grad);

/* ---- stage entry points (device pointers; used by callers that hold the
        OPD already, and by the parity tests) ---- */
/* (a) Ray trace of all layers for WFS iwfs at frame isim into opd
   (device, nsa*nopd^2 FP32, overwritten). */
int shwfs_raytrace_dev(shwfs_ctx* ctx, int iwfs, int isim, float* opd);
/* (b)-(e) from a given OPD (device, nsa*nopd^2 FP32) and optional LLT OPD
   (device, llt_nx^2 FP32 or NULL).  ints (device, nsa*npix FP32) and grad
   (device, 2*nsa FP32) are overwritten; either may be NULL when not wanted,
   except that gradients need ints internally.  isim selects the noise
   counter; noise is added only if the WFS is noisy and add_noise != 0. */
int shwfs_ints_grad_dev(shwfs_ctx* ctx, int iwfs, int isim, const float* opd, const float* lltopd,
	float* ints, float* grad, int add_noise);
/* (e) alone: gradients (device, 2*nsa) from pixel intensities (device, nsa*npix). */
int shwfs_grad_dev(shwfs_ctx* ctx, int iwfs, const float* ints, float* grad);
/* Photon and read noise added in place to n pixel intensities on the device:
   the rule of addnoise (lib/libmisc.c:31-55), with the optional per-pixel
   arrays bkgrnd2, bkgrnd2c and qe (device, n FP32, or NULL) and excess < 1
   taken as 1.  The draws are those of the frame kernels (Poisson by
   inversion below a mean of 10, transformed rejection up to 200, the
   reference's Gaussian rule above), from the counter (seed, pixel index,
   stream, frame), so the result depends on nothing else.  n < 2^32. */
int shwfs_addnoise_dev(shwfs_ctx* ctx, float* ints, long n, const float* bkgrnd2, const float* bkgrnd2c,
	const float* qe, double bkgrnd, double bkgrndc, double rne, double excess, uint64_t seed, uint32_t stream,
	uint32_t frame);
/* ---- stage timing: CUDA events around every launch on the context stream,
        as the reference's ctoc instrumentation (cuda/math/common.h:233-267) ---- */
#define SHWFS_STAGE_RAYTRACE 0 /* (a) ray trace into the subaperture OPD */
#define SHWFS_STAGE_UPLINK 1   /* LLT ray trace and uplink OTF */
#define SHWFS_STAGE_INTS 2     /* (b)-(e) imaging (FFT form: with noise and gradients) */
#define SHWFS_STAGE_POST 3     /* (d)-(e) noise and gradients after the tensor-core imaging */
#define SHWFS_NSTAGE 4
int shwfs_profile_enable(shwfs_ctx* ctx, int enable);
/* Waits for queued work, then returns per stage the summed device time (ms)
   and the number of kernel launches since the previous read, and resets. */
int shwfs_profile_read(shwfs_ctx* ctx, double* ms, int* launches);

/* ---- tuning ---- */
#define SHWFS_NVARIANT 6 /* imaging-kernel variants: 0-2 full-spectrum transforms at a register cap
                            for 4, 5 or 6 blocks per SM; 3-5 the half-spectrum form at the same caps */
/* Times every imaging-kernel variant on nrep whole frames of WFS
   [iwfs0, iwfs1) (their powfs; device time of the frame on the context's
   stream) and keeps the fastest; *chosen receives its index. */
int shwfs_autotune(shwfs_ctx* ctx, int iwfs0, int iwfs1, int nrep, int* chosen);
/* Selects an imaging-kernel variant explicitly. */
int shwfs_set_variant(shwfs_ctx* ctx, int ipowfs, int variant);
/* Order of the pupils in a ray-trace launch.  AUTO interleaves pupils of the
   same size (subaperture-major, pupil fastest) when the screens exceed L2,
   so that a screen row their footprints share is fetched once, and keeps
   the listed order otherwise; LISTED and INTERLEAVED force one order.  The
   OPD is the same in every order. */
#define SHWFS_TRACE_AUTO 0
#define SHWFS_TRACE_LISTED 1
#define SHWFS_TRACE_INTERLEAVED 2
int shwfs_set_trace_order(shwfs_ctx* ctx, int order);

/* Bytes the context has copied host->device and device->host on the frame
   path (descriptor tables, gradients, intensities) since the previous call;
   resets the counters. */
int shwfs_copy_counters(shwfs_ctx* ctx, uint64_t* h2d, uint64_t* d2h);

/* ---- allocation-free frame (no counterpart in the reference) ----
   One frame of WFS iwfs -- ray trace, uplink OTF, imaging, noise,
   gradients -- that allocates no device memory: its scratch (OPD, LLT OPD,
   uplink OTF, launch descriptor) lives in one file-scope device array of
   about 4 MiB that every GPU loading the library keeps until exit.  For
   callers that cannot call cudaMalloc once running: real-time loops that
   forbid allocation after start-up (it can block and can fail), and hosts
   whose device memory belongs to their own pool.  ints (nsa*npix) and grad (2*nsa) are device
   pointers owned by the caller; either may be NULL, not both.  Limits: at
   most SHWFS_NOALLOC_MAX_NSA subapertures, each of 16x16 OPD points padded
   to a 32x32 FFT (the 32-point form, at most 128 pixels); any other powfs
   (64-point and larger FFTs, geometric sensors, dtrat > 1, sigmatch 2) is
   rejected with SHWFS_EINVAL before anything is launched.  The first call on a device
   looks up the array's device address (cudaGetSymbolAddress).  Calls share
   the array: calls whose work overlaps on the GPU race; queue them on one
   stream. */
#define SHWFS_NOALLOC_MAX_NSA 4096
int shwfs_frame_noalloc(shwfs_ctx* ctx, int iwfs, int isim, float* ints, float* grad);

/* ---- the frame's imaging as one persistent launch ----
   With on != 0, shwfs_frame_queue and shwfs_frame_graph run the imaging
   (field, FFTs, transfer functions, pixels, noise, gradients) of every powfs
   of the frame in one persistent launch over a work list of (WFS,
   subaperture, FFT size) items: groups of four 32-point images, tiles of the
   FFT-pass chain of the 128- and 256-point images (each pass waits, bounded,
   for its image's previous pass) and their pixel steps; ray traces and
   uplinks stay separate launches.  Replaces the reference's per-WFS launch
   chains and cuFFT plans (cuda/sim/wfsgrad.cu:483-745,
   cuda/sim/wfsinit.cu:321-342).  FFT form, dtrat 1, sigmatch 0/1, at most 4
   powfs; a frame with any other powfs runs the ordinary per-powfs launches.
   slices (0 keeps the current value, default 7): the 32-point groups are cut
   into that many slices placed between the passes of the large images;
   group (0 keeps the current value, default 4, at most 64): 32-point images
   per work item. */
int shwfs_set_worklist(shwfs_ctx* ctx, int on, int slices, int group);
/* Times nrep whole frames of WFS [iwfs0, iwfs1) with the per-powfs launches
   and with the work list at (slices, group) = (7, 4), (14, 4), (28, 4),
   (7, 8), and keeps the fastest; *choice receives 0 for the per-powfs
   launches, 1-4 for the work-list settings in that order.  The frames run as
   CUDA graphs (shwfs_frame_graph; stream frames while stage profiling is on). */
int shwfs_autotune_frame(shwfs_ctx* ctx, int iwfs0, int iwfs1, int nrep, int* choice);
/* With on != 0 (the default), a frame of several powfs runs each powfs whose
   images per frame are fewer than the largest powfs's on a branch stream of
   the device's greatest priority, so their chains of small launches start as
   the large imaging kernel's blocks retire; with 0 every branch has the
   default priority.  Synchronises the context; the branches and the frame
   graph are made again by the next frame.  Results do not depend on it. */
int shwfs_set_branch_priority(shwfs_ctx* ctx, int on);
/* Stream priority of the context's stream (CUDA's scale: lower numbers run
   first; clamped to the device's range, 0 the default; the context's uplink
   stream stays at the greatest priority).  Synchronises the context and makes
   its streams again: shwfs_stream returns the new handle.
   A server of many contexts on one GPU uses it to let some contexts' blocks
   reach the SMs first.  Results do not depend on it. */
int shwfs_set_stream_priority(shwfs_ctx* ctx, int priority);

/* Synchronise the context stream; returns the first error of queued work. */
int shwfs_sync(shwfs_ctx* ctx);
/* The CUDA stream the context launches on (cudaStream_t as void*). */
void* shwfs_stream(shwfs_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
