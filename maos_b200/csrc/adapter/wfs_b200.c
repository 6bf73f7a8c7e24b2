/*
 * Adapter from MAOS's GPU wavefront-sensor seam to libshwfs_b200.
 *
 * This file belongs in the MAOS tree (beside cuda/sim/wfsgrad.cu) and is compiled against
 * the headers under maos/ and linked with -lshwfs_b200. It defines the C-linkage functions that the simulator
 * calls when gpu.wfs is set (cuda/sim/gpu_sim.h:39-49; selected in maos/sim_utils.c:1497-1504),
 * so maos.c's time loop is unchanged:
 *
 *   gpu_wfsgrad_init        cuda/sim/wfsinit.cu:159   powfs and WFS descriptors, geometry,
 *                                                     pixel maps, DTF/ETF, LLT, matched filters
 *   gpu_wfsgrad_update_etf  cuda/sim/wfsinit.cu:32    etfsim / etfsim2 slots, interpolation period
 *   gpu_wfsgrad_update_ref  cuda/sim/wfsinit.cu:107   matched filters and i0 sums
 *   gpu_wfsgrad_seeding     cuda/sim/wfsinit.cu:532   one lrand() per WFS
 *   gpu_atm2gpu             cuda/sim/atm.cu:106       turbulence screens
 *   gpu_wfsgrad_queue       cuda/sim/wfsgrad.cu:483   queue the frame of info->start..end
 *   gpu_wfsgrad_sync        cuda/sim/wfsgrad.cu:747   gradients into simu->gradcl
 *   gpu_dmreal2gpu          cuda/sim/atm.cu:315       DM surfaces, subtracted in closed loop
 *   gpu_wfssurf2gpu         cuda/sim/wfsinit.cu:514   NCPA surfaces (powfs.opdadd)
 *   gpu_wfs_init_sim, gpu_save_pistat: no device state to reset; pistatout is refused.
 *   gpu_dmproj2gpu: DM-projected turbulence (idealwfs, wfsalias) is refused.
 *   gpu_perfevl_init, gpu_perfevl_init_sim, gpu_perfevl_queue, gpu_perfevl_sync
 *                           cuda/sim/perfevl.cu: the open-loop science evaluation (olep, olmp
 *                           and the PSF sums); DM terms are refused.
 *
 * The reference aborts on errors (error()); a nonzero status from the library is reported the
 * same way, with the library's message.  Options of the reference's WFS path that the library
 * does not serve (more than SHWFS_MAX_BANDS + 1 wavelengths, sodium sublayers, per-WFS amplitude maps, cubic DMs,
 * MOAO, field stops, dithering, ...) are refused with error() at gpu_wfsgrad_init, so the
 * adapter never returns gradients that differ from MAOS's in silence. One context serves every WFS. The simulator queues and
 * syncs WFS from several host threads at once, and calls on one context must not overlap, so
 * every call goes through one mutex.
 */
#include <pthread.h>
#include <string.h>
#include "gpu_sim.h"
#include "shwfs_b200.h"
#include "shwfs_evl.h"

static shwfs_ctx* g_ctx;
static int g_ipowfs[64];   /* MAOS ipowfs -> context powfs (physical optics, or the geometric sensor) */
static int g_ipowfs_geo[64];/* MAOS ipowfs -> context geometric powfs before phystep, or -1 */
static int g_band[64][SHWFS_MAX_BANDS+1];/* MAOS ipowfs, wavelength -> context powfs of that band */
static int* g_wfs_phy;     /* MAOS iwfs -> context WFS with physical optics, or -1 */
static int* g_wfs_geo;     /* MAOS iwfs -> context geometric WFS, or -1 */
static int* g_wfs_cur;     /* MAOS iwfs -> the context WFS its last queued frame ran, or -1 */
static int g_nwfs;
static int g_ndm;          /* mirror grids held by the context (gpu_dmreal2gpu) */
static pthread_mutex_t g_lock=PTHREAD_MUTEX_INITIALIZER;

static shwfs_ctx* g_evl;   /* science path (gpu_perfevl_*): a context of its own */
static double* g_evl_wfe;  /* nevl x 3 {PR, TT, PTTR} of the last synced frame */
static double* g_evl_coeff;/* nevl x 3 {piston, tip, tilt} */
static int g_evl_synced=1; /* the queued frame's results are in g_evl_wfe/coeff */

static void chk_ctx(const shwfs_ctx* ctx, int rc, const char* what){
	if(rc) error("shwfs %s: %s\n", what, shwfs_last_error(ctx));
}
static void chk(int rc, const char* what){ chk_ctx(g_ctx, rc, what); }

/* dtf.si (npix x notf^2, CSC, bilinear: at most four entries per pixel row) -> 4-tap map */
static void si_taps(const dsp* si, int* idx, double* wt){
	const long npix=si->nx;
	for(long i=0; i<npix*4; i++){ idx[i]=-1; wt[i]=0; }
	int* k=mycalloc(npix, int);
	for(long ic=0; ic<si->ny; ic++){
		for(long j=si->pp[ic]; j<si->pp[ic+1]; j++){
			const long p=si->pi[j];
			if(k[p]>=4) error("shwfs: pixel %ld has more than four taps\n", p);
			idx[4*p+k[p]]=(int)ic; wt[4*p+k[p]]=si->px[j]; k[p]++;
		}
	}
	free(k);
}

/* etf.etf is a cell of nsa (x 1 or x nllt) notf x notf complex arrays; pack the first LLT's
   column subaperture-major, as shwfs_powfs_set_etf takes it. */
static void set_etf(const powfs_t* p, int ipl, const etf_t* etf, int slot){
	const long nsa=p->saloc->nloc, n2=(long)p->notfx*p->notfy;
	cmat* e=cnew(n2, nsa);
	for(long isa=0; isa<nsa; isa++) memcpy(PCOL(e, isa), P(P(etf->etf, isa, 0)), sizeof(comp)*n2);
	chk(shwfs_powfs_set_etf(g_ctx, ipl, (const double*)P(e), slot), "set_etf");
	cfree(e);
}

/* Wavelength iwvl's pixel map and ETF (LGS) or DTF nominal (powfs.dtf[iwvl], etfsim[iwvl])
   into context powfs ipl. */
static void load_band_data(const powfs_t* p, int iwvl, int ipl){
	/* dtf.si and dtf.nominal: one map shared by every subaperture, or one per subaperture
	   (lib/mkdtf.c:116-161: radpix or pixoffx) */
	const dspcell* si=p->dtf[iwvl].si;
	const long nmap=PN(si);
	const long npix=(long)p->pixpsax*p->pixpsay;
	int* idx=mymalloc(nmap*npix*4, int);
	double* wt=mymalloc(nmap*npix*4, double);
	for(long m=0; m<nmap; m++) si_taps(P(si, m), idx+m*npix*4, wt+m*npix*4);
	chk(shwfs_powfs_set_simap(g_ctx, ipl, idx, wt, (int)nmap), "set_simap");
	free(idx); free(wt);
	if(p->llt){
		set_etf(p, ipl, &p->etfsim[iwvl], 0);
	}else{
		/* nominal is real-valued in MAOS's FFT layout */
		const dcell* nom=p->dtf[iwvl].nominal;
		const long nn=PN(nom), n2=(long)p->notfx*p->notfy;
		dmat* all=dnew(n2, nn);
		for(long m=0; m<nn; m++) memcpy(PCOL(all, m), P(P(nom, m)), sizeof(real)*n2);
		chk(shwfs_powfs_set_nominal(g_ctx, ipl, P(all), (int)nn), "set_nominal");
		dfree(all);
	}
}

/* intstat->mtche is nsa x nwfs cells of 2 x npix; pack the WFS's column subaperture-major. */
static void set_mtche(const parms_t* parms, const powfs_t* p, int ip, int iwfs){
	const intstat_t* st=p->intstat;
	if(!st || !st->mtche || g_wfs_phy[iwfs]<0) return;
	const long wfsind=P(parms->powfs[ip].wfsind, iwfs);
	const long nsa=p->saloc->nloc, npix=(long)p->pixpsax*p->pixpsay;
	const long icol=NY(st->mtche)>1?wfsind:0;
	dmat* mt=dnew(2*npix, nsa);
	for(long isa=0; isa<nsa; isa++) memcpy(PCOL(mt, isa), P(P(st->mtche, isa, icol)), sizeof(real)*2*npix);
	const long ii0=NY(st->i0sum)>1?wfsind:0;
	chk(shwfs_wfs_set_mtche(g_ctx, g_wfs_phy[iwfs], P(mt), PCOL(st->i0sum, ii0), P(st->i0sumsum, ii0)),
		"set_mtche");
	dfree(mt);
}

/* Options of the reference's WFS path that this library does not serve: refused at set-up, so
   that a run never returns gradients that differ from MAOS's without an error. */
static void refuse_unsupported(const parms_t* parms, const powfs_t* powfs){
	if(parms->sim.idealwfs || parms->sim.wfsalias)
		error("shwfs: sim.idealwfs/sim.wfsalias (DM-projected turbulence) are not supported\n");
	if(parms->atm.dtrat>0) error("shwfs: atm.dtrat (screens played back in time) is not supported\n");
	if(parms->tomo.ahst_idealngs) error("shwfs: tomo.ahst_idealngs is not supported\n");
	for(int idm=0; idm<parms->ndm; idm++){
		if(parms->dm[idm].iac) error("shwfs: DM %d uses a cubic influence function (dm.iac); only linear DMs\n", idm);
	}
	for(int ip=0; ip<parms->npowfs; ip++){
		const powfs_cfg_t* pc=&parms->powfs[ip];
		const powfs_t* p=&powfs[ip];
		if(pc->type!=WFS_SH) error("shwfs: powfs %d is not a Shack-Hartmann WFS\n", ip);
		if(pc->nwvl>SHWFS_MAX_BANDS+1) error("shwfs: powfs %d has %d wavelengths; at most %d\n", ip, pc->nwvl,
			SHWFS_MAX_BANDS+1);
		/* the weights of the further wavelengths belong to the band, shared by the powfs' WFS */
		for(int jw=1; jw<pc->nwfs; jw++){
			const dmat* w0=parms->wfs[P(pc->wfs, 0)].wvlwts, * wj=parms->wfs[P(pc->wfs, jw)].wvlwts;
			for(int iwvl=1; iwvl<pc->nwvl; iwvl++)
				if(P(wj, iwvl)!=P(w0, iwvl))
					error("shwfs: powfs %d: WFS weights of wavelength %d differ between WFS\n", ip, iwvl);
		}
		if(pc->moao>-1) error("shwfs: powfs %d uses MOAO\n", ip);
		if(pc->fieldstop>0) error("shwfs: powfs %d has a field stop\n", ip);
		if(pc->dither) error("shwfs: powfs %d dithers\n", ip);
		if(pc->pistatout || pc->psfout) error("shwfs: powfs %d asks for pistatout/psfout diagnostics\n", ip);
		if(PN(p->amp)>1 || (p->saa && PN(p->saa)>1))
			error("shwfs: powfs %d has one amplitude map per WFS (misregistration); one shared map only\n", ip);
		if(pc->llt){
			if(pc->llt->nhs>1) error("shwfs: powfs %d simulates %d sodium sublayers (llt.nhs)\n", ip, pc->llt->nhs);
			if(PN(pc->llt->ox)>1) error("shwfs: powfs %d has %ld launch telescopes; one only\n", ip, PN(pc->llt->ox));
			if(p->llt && p->llt->ncpa) error("shwfs: powfs %d has an LLT surface (llt.ncpa)\n", ip);
		}
		if(pc->usephy){
			if(pc->phytype_sim!=PTYPE_MF && pc->phytype_sim!=PTYPE_COG)
				error("shwfs: powfs %d gradient type %d; matched filter or CoG only\n", ip, pc->phytype_sim);
			for(int iwvl=0; iwvl<pc->nwvl; iwvl++){
				const dtf_t* dtf=&p->dtf[iwvl];
				if(NY(dtf->si)>1 || NY(dtf->nominal)>1)
					error("shwfs: powfs %d has pixel maps per WFS (pixoffx/pixoffy per WFS)\n", ip);
			}
		}
	}
}

/* The physical-optics powfs of MAOS powfs ip; *ipl receives its index. */
static void add_phy_powfs(const parms_t* parms, const powfs_t* p, int ip, int* ipl){
	const powfs_cfg_t* pc=&parms->powfs[ip];
	const int llt=p->llt!=NULL;
	shwfs_powfs_desc d={
		.nsa=(int)p->saloc->nloc, .nopd=(int)p->pts->nxsa, .embfac=pc->embfac,
		.notf=p->notfx, .pixpsax=p->pixpsax, .pixpsay=p->pixpsay,
		.pixthetax=pc->radpixtheta, .pixthetay=pc->pixtheta,
		.wvl=P(pc->wvl, 0), .dsa=p->pts->dsa, .dx=p->pts->dx,
		.areascale=p->areascale, .hs=pc->hs,
		.has_etf=llt, .has_llt=llt, .llt_nx=llt?(int)p->llt->pts->nxsa:0,
		.llt_ox=llt?P(pc->llt->ox, 0):0, .llt_oy=llt?P(pc->llt->oy, 0):0,
		.llt_origx=llt?p->llt->pts->origx[0]:0, .llt_origy=llt?p->llt->pts->origy[0]:0,
		.gradtype=pc->phytype_sim, .sigmatch=pc->sigmatch,
		.cogthres=pc->cogthres, .cogoff=pc->cogoff, .rne=pc->rne,
		.bkgrnd=pc->bkgrnd*pc->dtrat, .bkgrndc=pc->bkgrnd*pc->dtrat*pc->bkgrndc,
		.saat=pc->saat, .sigtot_cog=pc->siglev*pc->dtrat};
	chk(shwfs_powfs_add(g_ctx, &d, ipl), "powfs_add");
	chk(shwfs_powfs_set_geom(g_ctx, *ipl, p->pts->origx, p->pts->origy, P(P(p->amp, 0)), 1, P(P(p->saa, 0))),
		"set_geom");
	chk(shwfs_powfs_set_saasum(g_ctx, *ipl, P(p->saasum, 0)), "set_saasum");
	if(llt) chk(shwfs_powfs_set_lltamp(g_ctx, *ipl, P(p->llt->amp)), "set_lltamp");
	load_band_data(p, 0, *ipl);
	g_band[ip][0]=*ipl;
	/* further wavelengths (powfs.wvl[1..]): bands imaged from the same OPD, weighted by the
	   WFS's wvlwts (maos/wfsints.c:145-288) */
	for(int iwvl=1; iwvl<pc->nwvl; iwvl++){
		shwfs_powfs_desc db=d;
		db.wvl=P(pc->wvl, iwvl);
		const double wt=P(parms->wfs[P(pc->wfs, 0)].wvlwts, iwvl);
		chk(shwfs_powfs_add_band(g_ctx, *ipl, &db, wt, &g_band[ip][iwvl]), "powfs_add_band");
		load_band_data(p, iwvl, g_band[ip][iwvl]);
	}
	if(pc->dtrat>1) chk(shwfs_powfs_set_dtrat(g_ctx, *ipl, pc->dtrat), "set_dtrat");
}

/* The geometric sensor of MAOS powfs ip (gtype_sim: z-tilt, or G-tilt through powfs.GS0):
   the sensor itself when usephy is 0, else the gradients before phystep. */
static void add_geo_powfs(const parms_t* parms, const powfs_t* p, int ip, int* ipl){
	const powfs_cfg_t* pc=&parms->powfs[ip];
	const int gtype=pc->gtype_sim==GTYPE_Z?SHWFS_GRAD_ZTILT:SHWFS_GRAD_GTILT;
	const int llt=p->llt!=NULL;  /* its position centres the trombone focus (loc_add_focus_offset) */
	shwfs_powfs_desc d={.nsa=(int)p->saloc->nloc, .nopd=(int)p->pts->nxsa, .embfac=1, .notf=1,
		.dsa=p->pts->dsa, .dx=p->pts->dx, .areascale=p->areascale, .hs=pc->hs, .gradtype=gtype,
		.saat=pc->saat, .llt_ox=llt?P(pc->llt->ox, 0):0, .llt_oy=llt?P(pc->llt->oy, 0):0};
	chk(shwfs_powfs_add(g_ctx, &d, ipl), "powfs_add");
	chk(shwfs_powfs_set_geom(g_ctx, *ipl, p->pts->origx, p->pts->origy, P(P(p->amp, 0)), 1, P(P(p->saa, 0))),
		"set_geom");
	if(gtype==SHWFS_GRAD_GTILT){
		const dsp* gs0=p->GS0?P(p->GS0, 0):NULL;
		if(!gs0) error("shwfs: powfs %d uses G-tilt gradients but powfs.GS0 is not set\n", ip);
		chk(shwfs_powfs_set_gs0(g_ctx, *ipl, 0, gs0->nx, gs0->ny, gs0->pp, gs0->pi, gs0->px), "set_gs0");
	}
	if(pc->dtrat>1) chk(shwfs_powfs_set_dtrat(g_ctx, *ipl, pc->dtrat), "set_dtrat");
}

void gpu_wfsgrad_init(const parms_t* parms, const powfs_t* powfs){
	refuse_unsupported(parms, powfs);
	pthread_mutex_lock(&g_lock);
	if(g_ctx){ /* a new simulation in the same process */
		shwfs_destroy(g_ctx);
		g_ctx=NULL;
	}
	chk(shwfs_create(&g_ctx, 0), "create");
	if(parms->npowfs>64) error("shwfs: at most 64 powfs\n");
	g_ndm=0;
	for(int ip=0; ip<parms->npowfs; ip++){
		const powfs_cfg_t* pc=&parms->powfs[ip];
		g_ipowfs_geo[ip]=-1;
		if(pc->usephy){
			add_phy_powfs(parms, &powfs[ip], ip, &g_ipowfs[ip]);
			if(pc->phystep>0) add_geo_powfs(parms, &powfs[ip], ip, &g_ipowfs_geo[ip]);
		}else{
			add_geo_powfs(parms, &powfs[ip], ip, &g_ipowfs[ip]);
			g_ipowfs_geo[ip]=g_ipowfs[ip];
		}
	}
	free(g_wfs_phy); free(g_wfs_geo); free(g_wfs_cur);
	g_nwfs=parms->nwfs;
	g_wfs_phy=mymalloc(g_nwfs, int);
	g_wfs_geo=mymalloc(g_nwfs, int);
	g_wfs_cur=mymalloc(g_nwfs, int);
	for(int iwfs=0; iwfs<parms->nwfs; iwfs++){
		const int ip=parms->wfs[iwfs].powfs;
		const powfs_cfg_t* pc=&parms->powfs[ip];
		const wfs_cfg_t* wc=&parms->wfs[iwfs];
		const long wfsind=P(pc->wfsind, iwfs);
		g_wfs_phy[iwfs]=g_wfs_geo[iwfs]=g_wfs_cur[iwfs]=-1;
		if(pc->usephy){
			shwfs_wfs_desc w={.ipowfs=g_ipowfs[ip], .thetax=wc->thetax, .thetay=wc->thetay,
				.hs=wc->hs, .hc=wc->hc, .misregx=wc->misregx, .misregy=wc->misregy,
				.sigsim=wc->sigsim, .wvlwt=P(wc->wvlwts, 0), .noisy=pc->noisy};
			chk(shwfs_wfs_add(g_ctx, &w, &g_wfs_phy[iwfs]), "wfs_add");
			set_mtche(parms, &powfs[ip], ip, iwfs);
		}
		if(g_ipowfs_geo[ip]>=0){
			/* noise on geometric gradients only for a geometric sensor, not before phystep
			   (cuda/sim/wfsgrad.cu:709-712) */
			const int noisy=pc->noisy && !pc->usephy;
			shwfs_wfs_desc w={.ipowfs=g_ipowfs_geo[ip], .thetax=wc->thetax, .thetay=wc->thetay,
				.hs=wc->hs, .hc=wc->hc, .misregx=wc->misregx, .misregy=wc->misregy,
				.sigsim=wc->sigsim, .wvlwt=1, .noisy=noisy};
			chk(shwfs_wfs_add(g_ctx, &w, &g_wfs_geo[iwfs]), "wfs_add");
			const dmat* nea=powfs[ip].neasim?PR(powfs[ip].neasim, wfsind, 0):NULL;
			if(noisy && nea) chk(shwfs_wfs_set_neasim(g_ctx, g_wfs_geo[iwfs], P(nea)), "set_neasim");
		}
	}
	chk(shwfs_set_dt(g_ctx, parms->sim.dt), "set_dt");
	pthread_mutex_unlock(&g_lock);
}

void gpu_wfs_init_sim(const parms_t* parms, powfs_t* powfs){
	(void)parms; (void)powfs; /* intensities and gradients are formed afresh each frame */
}

void gpu_wfsgrad_update_etf(const parms_t* parms, const powfs_t* powfs, int ipowfs){
	const powfs_t* p=&powfs[ipowfs];
	if(!p->llt || !parms->powfs[ipowfs].usephy) return;
	pthread_mutex_lock(&g_lock);
	for(int iwvl=0; iwvl<parms->powfs[ipowfs].nwvl; iwvl++){
		const int ipl=g_band[ipowfs][iwvl];
		set_etf(p, ipl, &p->etfsim[iwvl], 0);
		if(p->etfsim2){
			set_etf(p, ipl, &p->etfsim2[iwvl], 1);
			/* the interpolation period as maos/wfsints.c:218 picks it */
			const int dtrat=parms->powfs[ipowfs].llt->coldtrat?parms->powfs[ipowfs].llt->coldtrat
				:parms->powfs[ipowfs].zoomdtrat;
			chk(shwfs_powfs_set_etf_dtrat(g_ctx, ipl, dtrat), "set_etf_dtrat");
		}else{
			/* slot 0 alone: no interpolation left over from an earlier pair */
			chk(shwfs_powfs_set_etf_dtrat(g_ctx, ipl, 0), "set_etf_dtrat");
		}
	}
	pthread_mutex_unlock(&g_lock);
}

void gpu_wfsgrad_update_ref(const parms_t* parms, const powfs_t* powfs, int ipowfs){
	pthread_mutex_lock(&g_lock);
	for(int jwfs=0; jwfs<parms->powfs[ipowfs].nwfs; jwfs++){
		const int iwfs=P(parms->powfs[ipowfs].wfs, jwfs);
		set_mtche(parms, &powfs[ipowfs], ipowfs, iwfs);
	}
	pthread_mutex_unlock(&g_lock);
}

void gpu_wfsgrad_seeding(const parms_t* parms, const powfs_t* powfs, rand_t* rstat){
	(void)powfs;
	pthread_mutex_lock(&g_lock);
	for(int iwfs=0; iwfs<parms->nwfs; iwfs++){
		const long seed=lrand(rstat); /* one draw per WFS, as cuda/sim/wfsinit.cu:536 */
		if(g_wfs_phy[iwfs]>=0) chk(shwfs_wfs_seed(g_ctx, g_wfs_phy[iwfs], seed), "seed");
		if(g_wfs_geo[iwfs]>=0) chk(shwfs_wfs_seed(g_ctx, g_wfs_geo[iwfs], seed), "seed");
	}
	pthread_mutex_unlock(&g_lock);
}

void gpu_atm2gpu(const mapcell* atm, const dmat* atmscale, const parms_t* parms, int iseed, int isim){
	(void)parms; (void)iseed; (void)isim;
	/* atmscale (atm.r0evolve) scales the screens frame by frame (cuda/sim/accphi.cu:155-156);
	   the library's layer weights are fixed per screen set. */
	if(atmscale) error("shwfs: atm.r0evolve (a per-frame atmscale) is not supported\n");
	const int n=(int)PN(atm);
	shwfs_layer_desc* L=mycalloc(n, shwfs_layer_desc);
	const double** s=mycalloc(n, const double*);
	for(int i=0; i<n; i++){
		const map_t* m=P(atm, i);
		L[i]=(shwfs_layer_desc){.nx=m->nx, .ny=m->ny, .dx=m->dx, .ox=m->ox, .oy=m->oy,
			.ht=m->ht, .vx=m->vx, .vy=m->vy, .alpha=1};
		s[i]=P(m);
	}
	pthread_mutex_lock(&g_lock);
	/* the WFS and the science contexts each keep the screens, as the reference keeps them on
	   every GPU that traces them */
	if(g_ctx) chk(shwfs_atm_set(g_ctx, n, L, s), "atm_set");
	if(g_evl) chk_ctx(g_evl, shwfs_atm_set(g_evl, n, L, s), "atm_set");
	pthread_mutex_unlock(&g_lock);
	free(L); free(s);
}

/* The DM surfaces embedded in square maps (simu->dmrealsq, NaN outside the actuators), once per
   step after the servo (maos/filter.c:561, maos/sim_utils.c:1268).  Subtracted from the OPD of
   every WFS in closed loop. */
void gpu_dmreal2gpu(mapcell* dmreal){
	if(!dmreal) return;
	const int n=(int)PN(dmreal);
	shwfs_layer_desc* L=mycalloc(n, shwfs_layer_desc);
	const double** s=mycalloc(n, const double*);
	for(int i=0; i<n; i++){
		const map_t* m=P(dmreal, i);
		if(m->iac) error("shwfs: DM %d uses a cubic influence function; only linear DMs\n", i);
		L[i]=(shwfs_layer_desc){.nx=m->nx, .ny=m->ny, .dx=m->dx, .ox=m->ox, .oy=m->oy, .ht=m->ht, .alpha=-1};
		s[i]=P(m);
	}
	pthread_mutex_lock(&g_lock);
	if(g_ctx){
		chk(shwfs_dm_set(g_ctx, n, L, s), "dm_set");
		g_ndm=n;
	}
	pthread_mutex_unlock(&g_lock);
	free(L); free(s);
}

void gpu_dmproj2gpu(mapcell* dmproj){
	(void)dmproj;
	error("shwfs: sim.idealwfs/sim.wfsalias (DM-projected turbulence) are not supported\n");
}

/* The terms MAOS adds to a WFS OPD besides the turbulence (maos/wfsgrad.c:200-262, 373-377;
   cuda/sim/wfsgrad.cu:548-605), for the frame of step isim. */
static void set_opd_terms(const sim_t* simu, int iwfs, int lib_wfs, int isim){
	const parms_t* parms=simu->parms;
	const int ip=parms->wfs[iwfs].powfs;
	const int CL=parms->sim.closeloop;
	const int llt=simu->powfs[ip].llt!=NULL;
	double ptt[3]={0, 0, 0};
	if(simu->telws){ /* wind shake */
		const real tmp=P(simu->telws, isim);
		const real angle=simu->winddir?P(simu->winddir, 0):0;
		ptt[1]+=tmp*cos(angle);
		ptt[2]+=tmp*sin(angle);
	}
	if(CL){
		if(simu->ttmreal){
			ptt[1]-=P(simu->ttmreal, 0);
			ptt[2]-=P(simu->ttmreal, 1);
		}
		if(simu->fsmreal && P(simu->fsmreal, iwfs) && !llt){
			ptt[1]-=P(P(simu->fsmreal, iwfs), 0);
			ptt[2]-=P(P(simu->fsmreal, iwfs), 1);
		}
	}
	double ftel=0, fllt=0;
	if(simu->telfocusreal) ftel=-P(P(simu->telfocusreal, 0), 0);
	if(llt && (simu->zoomint || simu->powfs[ip].focus)){
		fllt=simu->zoomint?zoomfocusadj((sim_t*)simu, iwfs):PR(simu->powfs[ip].focus, isim, P(parms->powfs[ip].wfsind, iwfs));
	}
	/* the uplink tip/tilt reaches only the physical-optics frame (the LLT OPD, maos/wfsgrad.c:373-377) */
	const int phy=lib_wfs==g_wfs_phy[iwfs];
	real lt[2]={0, 0};
	if(llt && phy) wfsgrad_llt_tt(&lt[0], &lt[1], (sim_t*)simu, iwfs, isim);
	const double lltptt[2]={lt[0], lt[1]};
	chk(shwfs_wfs_set_opd_terms(g_ctx, lib_wfs, CL && g_ndm>0, ptt, ftel, fllt, (llt && phy)?lltptt:NULL),
		"set_opd_terms");
}

void* gpu_wfsgrad_queue(thread_t* info){
	sim_t* simu=(sim_t*)info->data;
	const parms_t* parms=simu->parms;
	const int isim=simu->wfsisim;
	pthread_mutex_lock(&g_lock);
	for(int iwfs=info->start; iwfs<info->end; iwfs++){
		const int ip=parms->wfs[iwfs].powfs;
		const powfs_cfg_t* pc=&parms->powfs[ip];
		g_wfs_cur[iwfs]=-1;
		if(isim<pc->step) continue; /* the WFS starts at powfs.step (cuda/sim/wfsgrad.cu:492) */
		const int do_phy=pc->usephy && isim>=pc->phystep;
		const int lw=do_phy?g_wfs_phy[iwfs]:g_wfs_geo[iwfs];
		set_opd_terms(simu, iwfs, lw, isim);
		chk(shwfs_frame_queue(g_ctx, isim, lw, lw+1), "frame_queue");
		g_wfs_cur[iwfs]=lw;
	}
	pthread_mutex_unlock(&g_lock);
	return NULL;
}

/* Gradients of the frame into simu->gradcl on the WFS's output frames ((isim+1) mod dtrat = 0,
   cuda/sim/wfsgrad.cu:747-776); other frames leave it as it was. */
void gpu_wfsgrad_sync(sim_t* simu, int iwfs){
	const int ip=simu->parms->wfs[iwfs].powfs;
	const int dtrat=simu->parms->powfs[ip].dtrat;
	pthread_mutex_lock(&g_lock);
	const int lw=g_wfs_cur[iwfs];
	if(lw>=0 && (simu->wfsisim+1)%dtrat==0){
		dmat** pg=&P(simu->gradcl, iwfs);
		if(!*pg) *pg=dnew(simu->powfs[ip].saloc->nloc*2, 1);
		chk(shwfs_frame_sync(g_ctx, lw, P(*pg), NULL), "frame_sync");
	}else if(lw>=0){
		chk(shwfs_sync(g_ctx), "sync");
	}
	pthread_mutex_unlock(&g_lock);
}

void gpu_save_pistat(sim_t* simu){
	(void)simu; /* pistatout is refused at set-up */
}

/* NCPA surfaces of every WFS (powfs.opdadd, cuda/sim/wfsinit.cu:514-524). */
void gpu_wfssurf2gpu(const parms_t* parms, powfs_t* powfs){
	pthread_mutex_lock(&g_lock);
	for(int iwfs=0; iwfs<parms->nwfs; iwfs++){
		const int ip=parms->wfs[iwfs].powfs;
		const int wfsind=P(parms->powfs[ip].wfsind, iwfs);
		const dmat* add=powfs[ip].opdadd?P(powfs[ip].opdadd, wfsind):NULL;
		if(g_wfs_phy[iwfs]>=0) chk(shwfs_wfs_set_opdadd(g_ctx, g_wfs_phy[iwfs], add?P(add):NULL), "set_opdadd");
		if(g_wfs_geo[iwfs]>=0) chk(shwfs_wfs_set_opdadd(g_ctx, g_wfs_geo[iwfs], add?P(add):NULL), "set_opdadd");
	}
	pthread_mutex_unlock(&g_lock);
}

/* ---- science path, open loop (cuda/sim/perfevl.cu) ---- */

void gpu_perfevl_init(const parms_t* parms, aper_t* aper){
	const int nevl=parms->evl.nevl;
	if(parms->ndm>0) error("shwfs: the science path has no DM terms (parms->ndm=%d)\n", parms->ndm);
	if(parms->evl.nmod!=3) error("shwfs: the science path forms piston/tip/tilt only (evl.nmod=%d)\n",
		parms->evl.nmod);
	for(int i=1; i<nevl; i++){
		if(P(parms->evl.pttr, i)!=P(parms->evl.pttr, 0)) error("shwfs: evl.pttr must be the same for every direction\n");
	}
	pthread_mutex_lock(&g_lock);
	if(g_evl){
		shwfs_destroy(g_evl);
		g_evl=NULL;
	}
	chk_ctx(g_evl, shwfs_create(&g_evl, 0), "create");
	chk_ctx(g_evl, shwfs_set_dt(g_evl, parms->sim.dt), "set_dt");
	const loc_t* locs=aper->locs;
	chk_ctx(g_evl, shwfs_evl_set_aper(g_evl, locs->nloc, locs->locx, locs->locy, locs->dx, P(aper->amp)),
		"evl_set_aper");
	for(int ievl=0; ievl<nevl; ievl++){
		int k;
		chk_ctx(g_evl, shwfs_evl_add_dir(g_evl, P(parms->evl.thetax, ievl), P(parms->evl.thetay, ievl),
			P(parms->evl.hs, ievl), &k), "evl_add_dir");
	}
	if(parms->evl.psfmean && aper->locfft){
		const int nwvl=parms->evl.nwvl;
		int* nembed=mycalloc(nwvl, int);
		int* psfsize=mycalloc(nwvl, int);
		for(int i=0; i<nwvl; i++){
			nembed[i]=(int)P(aper->locfft->nembed, i);
			psfsize[i]=(int)P(parms->evl.psfsize, i);
		}
		chk_ctx(g_evl, shwfs_evl_set_psf(g_evl, nwvl, P(parms->evl.wvl), nembed, psfsize,
			(int)P(parms->evl.pttr, 0)), "evl_set_psf");
		free(nembed);
		free(psfsize);
	}
	free(g_evl_wfe);
	free(g_evl_coeff);
	g_evl_wfe=mycalloc(3*nevl, double);
	g_evl_coeff=mycalloc(3*nevl, double);
	g_evl_synced=1;
	pthread_mutex_unlock(&g_lock);
}

void gpu_perfevl_init_sim(const parms_t* parms, aper_t* aper){
	(void)parms; (void)aper;
	pthread_mutex_lock(&g_lock);
	if(g_evl) chk_ctx(g_evl, shwfs_evl_psf_reset(g_evl), "evl_psf_reset");
	pthread_mutex_unlock(&g_lock);
}

/* The simulator splits the directions over threads (info->start..end). One queue call runs every
   direction, so the thread holding direction 0 queues the frame; the syncs of all threads follow
   the queues (maos/sim.c runs perfevl_pre before perfevl_post). */
void* gpu_perfevl_queue(thread_t* info){
	sim_t* simu=(sim_t*)info->data;
	const parms_t* parms=simu->parms;
	if(info->start!=0) return NULL;
	const int do_psf=parms->evl.psfmean && simu->perfisim>=parms->evl.psfisim;
	pthread_mutex_lock(&g_lock);
	chk_ctx(g_evl, shwfs_evl_queue(g_evl, simu->perfisim, do_psf), "evl_queue");
	g_evl_synced=0;
	pthread_mutex_unlock(&g_lock);
	return NULL;
}

/* Open-loop results of frame perfisim into simu->olep (PR, TT, PTTR) and simu->olmp (piston,
   tip, tilt), column perfisim, for the thread's directions. */
void* gpu_perfevl_sync(thread_t* info){
	sim_t* simu=(sim_t*)info->data;
	const int isim=simu->perfisim;
	pthread_mutex_lock(&g_lock);
	if(!g_evl_synced){
		chk_ctx(g_evl, shwfs_evl_sync(g_evl, g_evl_wfe, g_evl_coeff), "evl_sync");
		g_evl_synced=1;
	}
	for(long ievl=info->start; ievl<info->end; ievl++){
		real* pe=PCOL(P(simu->olep, ievl), isim);
		real* pm=PCOL(P(simu->olmp, ievl), isim);
		for(int k=0; k<3; k++){
			pe[k]=g_evl_wfe[3*ievl+k];
			pm[k]=g_evl_coeff[3*ievl+k];
		}
	}
	pthread_mutex_unlock(&g_lock);
	return NULL;
}
