/*
 * Test-oracle driver around the reference's OWN C code for the
 * Shack-Hartmann physical-optics path.  Built by oracle/Makefile into
 * oracle/_ref/libmaosref.so from the sources under the reference tree (which
 * are compiled in place, never copied).  Test infrastructure only: the
 * product never links or calls it.
 *
 * It includes the reference's maos/powfs.c so that the static setup routines
 * (setup_shwfs_geom, setup_shwfs_prep_phy, setup_shwfs_dtf, setup_shwfs_etf,
 * setup_powfs_llt, setup_shwfs_phygrad) run exactly as MAOS runs them, and it
 * then calls the reference's per-frame routines:
 *   wfsints()      maos/wfsints.c:79
 *   shwfs_grad()   maos/utils.c:983
 *   addnoise()     lib/libmisc.c:31
 *   prop()         lib/accphi.c:223 (prop_grid_pts, lib/accphi_grid_do.c:408)
 *   genscreen      lib/turbulence.c:214 (via genatm_simple, lib/turbulence.c:371)
 *
 * The flat API below (oref_*) is what tests/ and bench.py's CPU-baseline leg
 * call through ctypes.  Arrays cross it as plain double pointers in MAOS
 * column-major order.
 */
#include "powfs.c"  /* reference maos/powfs.c, for its static setup routines */
#include <omp.h>
/* maos/wfsints.c:79; declared in the reference only inside its simulator headers */
void* wfsints(thread_t* thread_data);

typedef struct oref_cfg_t{
	double D, Din;        /* telescope diameter and central obstruction (m) */
	int amp_binary;       /* 1: binary annular pupil map sampled on the OPD grid */
	int order;            /* subapertures across the pupil */
	double dsa;           /* subaperture size (m) */
	double dx;            /* OPD sampling (m) */
	double saat;          /* subaperture area threshold */
	int embfac;           /* embedding factor, normally 2 */
	int notf;             /* OTF size; 0 = automatic */
	int pixpsa;           /* pixels per subaperture side */
	double pixtheta;      /* pixel size (rad) */
	double pixblur;       /* pixel blur sigma (fraction of pixel) */
	double wvl;           /* wavelength (m) */
	double hs;            /* guide star range (m); INFINITY for NGS */
	double siglev;        /* photons per subaperture per frame */
	double rne;           /* read noise (e-) */
	double bkgrnd;        /* background (e-/pixel/frame) */
	double bkgrndc;       /* calibrated fraction of background */
	int phytype;          /* 1: matched filter, 2: CoG */
	int sigmatch;         /* 0,1,2 */
	int mtchcr;           /* matched filter constraint */
	double cogthres, cogoff;
	double r0, L0;        /* turbulence used for the matched filter i0 */
	int has_llt;
	double llt_d, llt_widthp, llt_ox, llt_oy;
	int na_n;             /* sodium profile samples (evenly spaced) */
	const double* na_h;   /* altitude (m) */
	const double* na_p;   /* strength; sums to the signal scaling */
	int nwfs;
	const double* thetax; /* rad */
	const double* thetay; /* rad */
	int nthread;          /* NTHREAD for the reference's own threading */
	int nwvl;             /* wavelengths (0 or 1: wvl alone) */
	const double* wvls;   /* nwvl wavelengths (m) */
	const double* wvlwts; /* nwvl weights */
}oref_cfg_t;

static parms_t* g_parms=NULL;
static dsp* g_gs0=NULL;  /* G-tilt operator of the current powfs, made on first use */
static powfs_t* g_powfs=NULL;
static dmat* g_wvl=NULL;

static lmat* lvec(long n, long start){
	lmat* v=lnew(n, 1);
	for(long i=0; i<n; i++) P(v, i)=start+i;
	return v;
}

/* Builds parms_t/powfs_t for one powfs with cfg->nwfs WFS and runs the
   reference's SH setup. Returns the number of valid subapertures. */
void oref_cl_set(int ndm, const double* const* surf, const long* nx, const long* ny, const double* dx,
	const double* ox, const double* oy, const double* ht, int use_dm, const double* ptt, double focus_tel,
	double focus_llt, const double* lltptt, const double* opdadd);
static int g_iwvl;
int oref_setup(const oref_cfg_t* c){
	g_iwvl=0;
	dspfree(g_gs0);
	g_gs0=NULL;
	/* a new powfs starts with no closed-loop terms */
	oref_cl_set(0, NULL, NULL, NULL, NULL, NULL, NULL, NULL, 0, NULL, 0, 0, NULL, NULL);
	if(!global) global=mycalloc(1, global_t);
	NTHREAD=c->nthread>0?c->nthread:1;
	omp_set_num_threads(NTHREAD);
	parms_t* parms=g_parms=mycalloc(1, parms_t);
	parms->npowfs=1;
	parms->nwfs=c->nwfs;
	parms->powfs=mycalloc(1, powfs_cfg_t);
	parms->wfs=mycalloc(c->nwfs, wfs_cfg_t);
	parms->aper.d=c->D;
	parms->aper.din=c->Din;
	parms->aper.misreg=dnew(2, 1);
	parms->sim.dt=1./800;
	parms->sim.dtref=parms->sim.dt;
	parms->sim.za=0;
	parms->sim.htel=0;
	parms->dbg.wfslinearity=-1;
	parms->save.gradnf=lnew(c->nwfs, 1);
	powfs_cfg_t* p=parms->powfs;
	{
		/* powfs.wvl, powfs.wvlwts and wvlmean as maos/parms.c:266-283 reads them */
		const int nwvl=(c->nwvl>1&&c->wvls)?c->nwvl:1;
		g_wvl=dnew(nwvl, 1);
		p->wvlwts=dnew(nwvl, 1);
		real wm=0;
		for(int i=0; i<nwvl; i++){
			P(g_wvl, i)=nwvl>1?c->wvls[i]:c->wvl;
			P(p->wvlwts, i)=(nwvl>1&&c->wvlwts)?c->wvlwts[i]:1;
			wm+=P(g_wvl, i);
		}
		p->wvl=g_wvl;
		p->nwvl=nwvl;
		p->wvlmean=wm/nwvl;
	}
	p->order=c->order;
	p->dsa=c->dsa;
	p->dx=c->dx;
	p->saat=c->saat;
	p->safill2d=1;
	p->embfac=c->embfac;
	p->notf=c->notf;
	p->pixpsa=c->pixpsa;
	p->pixtheta=c->pixtheta;
	p->radpixtheta=c->pixtheta;
	p->pixblur=c->pixblur;
	p->hs=c->hs;
	p->siglev=c->siglev;
	p->rne=c->rne;
	p->bkgrnd=c->bkgrnd;
	p->bkgrndc=c->bkgrndc;
	p->phytype_recon=c->phytype;
	p->phytype_sim=c->phytype;
	p->phyusenea=1;
	p->sigmatch=c->sigmatch;
	p->mtchcr=c->mtchcr;
	p->cogthres=c->cogthres;
	p->cogoff=c->cogoff;
	p->r0=c->r0;
	p->L0=c->L0;
	p->dtrat=1;
	p->moao=-1;   /* no MOAO (the configuration default) */
	p->usephy=1;
	p->noisy=1;
	p->nwfs=c->nwfs;
	p->wfs=lvec(c->nwfs, 0);
	p->wfsind=lvec(c->nwfs, 0);
	p->siglevs=dnew(1, 1); P(p->siglevs, 0)=c->siglev;
	for(int iwfs=0; iwfs<c->nwfs; iwfs++){
		wfs_cfg_t* w=&parms->wfs[iwfs];
		w->powfs=0;
		w->thetax=c->thetax?c->thetax[iwfs]:0;
		w->thetay=c->thetay?c->thetay[iwfs]:0;
		w->hs=c->hs;
		w->siglev=c->siglev;
		w->sigsim=c->siglev;
		w->wvlwts=dref(p->wvlwts);
	}
	if(c->has_llt){
		llt_cfg_t* l=p->llt=mycalloc(1, llt_cfg_t);
		l->d=c->llt_d;
		l->widthp=c->llt_widthp;
		l->ox=dnew(1, 1); P(l->ox, 0)=c->llt_ox;
		l->oy=dnew(1, 1); P(l->oy, 0)=c->llt_oy;
		l->misreg=dnew(2, 1);
		l->i=lnew(c->nwfs, 1); /* every WFS uses LLT 0 */
		l->nllt=1;
		l->nhs=1;
		l->na_interp=1;
		p->trs=1;
	}
	global->parms=parms;
	powfs_t* powfs=g_powfs=mycalloc(1, powfs_t);
	global->powfs=powfs;

	map_t* aper=NULL;
	if(c->amp_binary){
		/* Binary annulus on a grid whose nodes coincide with the OPD points,
		   so the bilinear sampling in mkamp() returns the node values. */
		const double dxo=c->dsa/(2*(int)round(0.5*c->dsa/c->dx));
		long n=(long)ceil(c->D/dxo)+4;
		aper=mapnew(n, n, dxo, dxo);
		double off=((c->order&1)?-0.5*c->dsa:0)+0.5*dxo;
		long k0=(long)ceil((0.5*c->D+2*dxo)/dxo);
		aper->ox=off-k0*dxo;
		aper->oy=off-k0*dxo;
		for(long iy=0; iy<n; iy++){
			double y=aper->oy+iy*dxo;
			for(long ix=0; ix<n; ix++){
				double x=aper->ox+ix*dxo;
				double r2=x*x+y*y;
				P(aper, ix, iy)=(r2<=0.25*c->D*c->D&&r2>=0.25*c->Din*c->Din)?1:0;
			}
		}
	}
	setup_shwfs_geom(powfs, parms, aper, 0);
	setup_shwfs_prep_phy(powfs, parms, 0);
	setup_shwfs_dtf(powfs, parms, 0);
	if(c->has_llt){
		dmat* na=dnew(c->na_n, 2);
		for(int i=0; i<c->na_n; i++){
			P(na, i, 0)=c->na_h[i];
			P(na, i, 1)=c->na_p[i];
		}
		powfs[0].sodium=dcellnew(1, 1);
		P(powfs[0].sodium, 0)=na;
		setup_shwfs_etf(powfs, parms, 0, 1, 0, 0, 0);
		setup_powfs_llt(powfs, parms, 0);
	}
	if(c->phytype==PTYPE_MF){
		setup_shwfs_phygrad(powfs, parms, 0);
	}
	mapfree(aper);
	return (int)powfs[0].saloc->nloc;
}

int oref_nsa(void){ return (int)g_powfs[0].saloc->nloc; }
/* The structures built by oref_setup and oref_atm_set, for the driver of the MAOS-side adapter
   (adapter_driver.c), which hands them to MAOS's GPU seam as the simulator does. */
parms_t* oref_parms(void){ return g_parms; }
powfs_t* oref_powfs(void){ return g_powfs; }
int oref_nopd(void){ return (int)g_powfs[0].pts->nxsa; }
int oref_notf(void){ return g_powfs[0].notfx; }
int oref_pixpsax(void){ return g_powfs[0].pixpsax; }
int oref_pixpsay(void){ return g_powfs[0].pixpsay; }
double oref_areascale(void){ return g_powfs[0].areascale; }
/* the wavelength whose DTF, pixel map and ETF the getters below return */
static int g_iwvl=0;
void oref_select_wvl(int iwvl){ g_iwvl=(iwvl>=0&&iwvl<g_parms->powfs[0].nwvl)?iwvl:0; }
double oref_dtheta(void){ return g_powfs[0].dtf[g_iwvl].dtheta; }
int oref_llt_nx(void){ return g_powfs[0].llt?(int)g_powfs[0].llt->pts->nxsa:0; }

static void copy_vec(double* out, const double* in, long n){ memcpy(out, in, sizeof(double)*n); }

void oref_get_saloc(double* x, double* y){
	long n=g_powfs[0].saloc->nloc;
	copy_vec(x, g_powfs[0].saloc->locx, n);
	copy_vec(y, g_powfs[0].saloc->locy, n);
}
void oref_get_ptsorig(double* x, double* y){
	long n=g_powfs[0].pts->nsa;
	for(long i=0; i<n; i++){ x[i]=g_powfs[0].pts->origx[i]; y[i]=g_powfs[0].pts->origy[i]; }
}
double oref_get_ptsdx(void){ return g_powfs[0].pts->dx; }
void oref_get_amp(double* amp){ dmat* a=P(g_powfs[0].amp, 0); copy_vec(amp, P(a), PN(a)); }
void oref_get_saa(double* saa){ dmat* a=P(g_powfs[0].saa, 0); copy_vec(saa, P(a), PN(a)); }
double oref_get_saasum(void){ return P(g_powfs[0].saasum, 0); }
/* nominal DTF (treated, peak in corner with chess pattern) for subaperture isa */
void oref_get_nominal(int isa, double* out){
	dcell* nom=g_powfs[0].dtf[g_iwvl].nominal;
	dmat* n=PN(nom)==1?P(nom, 0):P(nom, isa);
	copy_vec(out, P(n), PN(n));
}
/* pixel sampling matrix si (npix x notf^2) of subaperture isa, dense, column-major */
void oref_get_si_dense(int isa, double* out){
	dspcell* sis=g_powfs[0].dtf[g_iwvl].si;
	dsp* si=PN(sis)==1?P(sis, 0):P(sis, isa);
	long nr=si->nx, nc=si->ny;
	memset(out, 0, sizeof(double)*nr*nc);
	for(long ic=0; ic<nc; ic++){
		for(long k=si->pp[ic]; k<si->pp[ic+1]; k++){
			out[si->pi[k]+ic*nr]+=si->px[k];
		}
	}
}
/* ETF with the nominal fused in, subaperture isa, interleaved complex notf^2 */
void oref_get_etf(int isa, double* out){
	cmat* e=P(g_powfs[0].etfsim[g_iwvl].etf, isa, 0);
	copy_vec(out, (double*)P(e), 2*PN(e));
}
void oref_get_srot(double* out){ dmat* a=P(g_powfs[0].srot, 0); copy_vec(out, P(a), PN(a)); }
void oref_get_srsa(double* out){ dmat* a=P(g_powfs[0].srsa, 0); copy_vec(out, P(a), PN(a)); }
void oref_get_lltamp(double* out){ copy_vec(out, P(g_powfs[0].llt->amp), PN(g_powfs[0].llt->amp)); }
/* matched filter of subaperture isa: 2 x npix column-major */
void oref_get_mtche(int isa, double* out){
	dmat* m=P(g_powfs[0].intstat->mtche, isa, 0);
	copy_vec(out, P(m), PN(m));
}
void oref_get_i0sum(double* out){
	dmat* s=g_powfs[0].intstat->i0sum;
	for(long i=0; i<NX(s); i++) out[i]=P(s, i, 0);
}
double oref_get_i0sumsum(void){ return P(g_powfs[0].intstat->i0sumsum, 0); }
/* The short-exposure PSF of subaperture isa (intstat->sepsf, gensepsf, lib/gensei.c:135-209):
   notf^2, peak in the centre. */
void oref_get_sepsf(int isa, double* out){
	const dmat* p=P(P(g_powfs[0].intstat->sepsf, 0, 0), isa);
	copy_vec(out, P(p), PN(p));
}
/* turbcov (lib/turbulence.c:400-435) of n separations r with rmax 0. */
void oref_turbcov(const double* r, long n, double r0, double L0, double* out){
	dmat* rr=dnew(n, 1);
	memcpy(P(rr), r, sizeof(double)*n);
	dmat* c=turbcov(rr, 0, r0, L0);
	copy_vec(out, P(c), n);
	dfree(c);
	dfree(rr);
}
void oref_get_i0(int isa, double* i0, double* gx, double* gy){
	intstat_t* st=g_powfs[0].intstat;
	copy_vec(i0, P(P(st->i0, isa, 0)), PN(P(st->i0, isa, 0)));
	if(gx) copy_vec(gx, P(P(st->gx, isa, 0)), PN(P(st->gx, isa, 0)));
	if(gy) copy_vec(gy, P(P(st->gy, isa, 0)), PN(P(st->gy, isa, 0)));
}

/* One WFS frame of wfsints() over subapertures [isa0, isa1), single thread.
   opd: nsa*nopd^2; lltopd: nlx^2 or NULL; ints: nsa*npix accumulated. */
void oref_wfsints(int iwfs, const double* opd, const double* lltopd, double* ints, int isa0, int isa1, int isim){
	const long nsa=g_powfs[0].saloc->nloc;
	const long nopd=g_powfs[0].pts->nxsa;
	const long npx=g_powfs[0].pixpsax, npy=g_powfs[0].pixpsay;
	dmat* dopd=dnew_do(nsa*nopd*nopd, 1, (double*)opd, 0);
	dmat* dllt=NULL;
	if(lltopd){
		long nlx=g_powfs[0].llt->pts->nxsa;
		dllt=dnew_do(nlx, nlx, (double*)lltopd, 0);
	}
	dcell* dints=dcellnew(nsa, 1);
	for(long isa=0; isa<nsa; isa++){
		P(dints, isa)=dnew_do(npx, npy, ints+isa*npx*npy, 0);
	}
	wfsints_t data={0};
	data.ints=dints;
	data.opd=dopd;
	data.lltopd=dllt;
	data.iwfs=iwfs;
	data.isim=isim;
	thread_t thd={0};
	thd.start=isa0;
	thd.end=isa1;
	thd.nthread=1;
	thd.data=&data;
	wfsints(&thd);
	dcellfree(dints);
	dfree(dopd);
	dfree(dllt);
}

/* Gradients of one WFS from ints (nsa*npix); grad: 2*nsa (x then y). */
void oref_shwfs_grad(int iwfs, const double* ints, double* grad){
	const long nsa=g_powfs[0].saloc->nloc;
	const long npx=g_powfs[0].pixpsax, npy=g_powfs[0].pixpsay;
	dmat** pints=mycalloc(nsa, dmat*);
	for(long isa=0; isa<nsa; isa++){
		pints[isa]=dnew_do(npx, npy, (double*)ints+isa*npx*npy, 0);
	}
	dmat* g=dnew_do(2*nsa, 1, grad, 0);
	shwfs_grad(&g, pints, g_parms, g_powfs, iwfs, g_parms->powfs[0].phytype_sim);
	for(long isa=0; isa<nsa; isa++) dfree(pints[isa]);
	free(pints);
	dfree(g);
}

/* Photon + read noise on ints (nsa*npix) with the reference's MT19937 stream. */
void oref_addnoise(double* ints, long n, unsigned int seed, double bkgrnd, double bkgrndc, double rne){
	rand_t rstat;
	seed_rand(&rstat, seed);
	dmat* a=dnew_do(n, 1, ints, 0);
	addnoise(a, &rstat, bkgrnd, bkgrndc, NULL, NULL, NULL, rne, 1.);
	dfree(a);
}

/* Ray trace one layer into the WFS OPD points (accumulates into opd). */
void oref_prop_layer(const double* screen, long nx, long ny, double dx, double ox, double oy, double ht,
	double thetax, double thetay, double hs, double shiftx, double shifty, double alpha, int wrap,
	double* opd, int isa0, int isa1){
	map_t* m=mapnew(nx, ny, dx, dx);
	memcpy(P(m), screen, sizeof(double)*nx*ny);
	m->ox=ox; m->oy=oy; m->ht=ht;
	prop_range(&(propdata_t){.mapin=m, .ptsout=g_powfs[0].pts, .phiout=opd, .alpha=alpha,
		.hs=hs, .thetax=thetax, .thetay=thetay, .shiftx=shiftx, .shifty=shifty, .wrap=wrap}, isa0, isa1);
	mapfree(m);
}
/* Ray trace one layer into the LLT pupil (nlx^2, accumulates) as maos/wfsgrad.c:337-365. */
void oref_prop_llt(const double* screen, long nx, long ny, double dx, double ox, double oy, double ht,
	double thetax, double thetay, double hs, double shiftx, double shifty, double* lltopd){
	map_t* m=mapnew(nx, ny, dx, dx);
	memcpy(P(m), screen, sizeof(double)*nx*ny);
	m->ox=ox; m->oy=oy; m->ht=ht;
	prop(&(propdata_t){.mapin=m, .ptsout=g_powfs[0].llt->pts, .phiout=lltopd, .alpha=1,
		.hs=hs, .thetax=thetax, .thetay=thetay, .shiftx=shiftx, .shifty=shifty, .wrap=1});
	mapfree(m);
}

/* The known-answer screen of test/cmocka_psd.c: genatm_simple(r0, L0, slope, dx, n, seed). */
void oref_genatm_simple(double r0, double L0, double slope, double dx, long n, unsigned int seed, double* out){
	dmat* s=genatm_simple(r0, L0, slope, dx, n, seed);
	copy_vec(out, P(s), PN(s));
	dfree(s);
}

/* Von Karman screens of nlayer layers with weights wt from one seed, made by the
   reference's genscreen (lib/turbulence.c:214, spect_screen_do :70-168): the
   layers come in pairs from one complex transform, every layer with outer
   scale L0.  out[i] receives the nx*ny values of layer i (x fastest). */
void oref_genscreen(int nlayer, long nx, long ny, double dx, double r0, double L0, const double* wt,
	unsigned int seed, double* const* out){
	rand_t rstat;
	seed_rand(&rstat, seed);
	real* w=mycalloc(nlayer, real);
	real* l0=mycalloc(nlayer, real);
	for(int i=0; i<nlayer; i++){ w[i]=wt[i]; l0[i]=L0; }
	genatm_t cfg={&rstat, w, r0, l0, dx, 0, 0, -11./3., nx, ny, nlayer, 0, 0, 0, 0};
	mapcell* screens=genscreen(&cfg);
	for(int i=0; i<nlayer; i++) copy_vec(out[i], P(P(screens, i)), nx*ny);
	cellfree(screens);
	free(w);
	free(l0);
}

/* Uniform and normal draws from the reference's RNG, for checking a restatement. */
void oref_rand_stream(unsigned int seed, long n, double* u, double* g, long* pois, double pois_mean){
	rand_t rstat;
	seed_rand(&rstat, seed);
	for(long i=0; i<n; i++){
		if(u) u[i]=randu(&rstat);
		if(g) g[i]=randn(&rstat);
		if(pois) pois[i]=randp(&rstat, pois_mean);
	}
}

/* The reference's multithreaded CPU frame for one WFS, as the MAOS time step
   runs it: wfsints over thread_prep(0,nsa,NTHREAD) (maos/sim_utils.c:1072-1079),
   then addnoise per subaperture and shwfs_grad.  Returns seconds spent. */
/* frame index passed to wfsints (ETF time interpolation, maos/wfsints.c:215-223) */
static int g_frame_isim=0;
double oref_frame_mt(int iwfs, const double* opd, const double* lltopd, double* ints, double* grad,
	unsigned int seed, int noisy){
	const long nsa=g_powfs[0].saloc->nloc;
	const long nopd=g_powfs[0].pts->nxsa;
	const long npx=g_powfs[0].pixpsax, npy=g_powfs[0].pixpsay;
	double t0=omp_get_wtime();
	dmat* dopd=dnew_do(nsa*nopd*nopd, 1, (double*)opd, 0);
	dmat* dllt=NULL;
	if(lltopd){
		long nlx=g_powfs[0].llt->pts->nxsa;
		dllt=dnew_do(nlx, nlx, (double*)lltopd, 0);
	}
	dcell* dints=dcellnew(nsa, 1);
	for(long isa=0; isa<nsa; isa++){
		P(dints, isa)=dnew_do(npx, npy, ints+isa*npx*npy, 0);
		dzero(P(dints, isa));
	}
	wfsints_t data={0};
	data.ints=dints;
	data.opd=dopd;
	data.lltopd=dllt;
	data.iwfs=iwfs;
	data.isim=g_frame_isim;
	thread_t* thd=thread_prep(0, nsa, NTHREAD, wfsints, &data);
	CALL_THREAD(thd, 1);
	free(thd);
	if(noisy){
		rand_t rstat;
		seed_rand(&rstat, seed);
		const real bkgrnd=g_parms->powfs[0].bkgrnd;
		const real bkgrndc=bkgrnd*g_parms->powfs[0].bkgrndc;
		for(long isa=0; isa<nsa; isa++){
			addnoise(P(dints, isa), &rstat, bkgrnd, bkgrndc, NULL, NULL, NULL, g_parms->powfs[0].rne, 1.);
		}
	}
	dmat* g=dnew_do(2*nsa, 1, grad, 0);
	shwfs_grad(&g, P(dints), g_parms, g_powfs, iwfs, g_parms->powfs[0].phytype_sim);
	double t1=omp_get_wtime();
	dfree(g);
	dcellfree(dints);
	dfree(dopd);
	dfree(dllt);
	return t1-t0;
}

/* The known-answer numbers of test/cmocka_psd.c for the screen
   genatm_simple(0.186, 0, -11/3, 1/64, 128, seed=1):
   out[0]=rms (nm), out[1]=psd2d_aniso integral (nm), out[2]=psd2d integral
   (nm), out[3]=fitted r0, out[4]=fitted slope, out[5]=sum(stfun)*1e9,
   out[6]=max(stfun)*1e13. */
void oref_kat_psd(double* out){
	dmat* screen=(dmat*)genatm_simple(0.186, 0, -11./3., 1./64., 128, 1);
	dmat* psd=psd2d_aniso(screen, 1./64.);
	out[1]=sqrt(psd_inte2(psd))*1e9;
	dfree(psd);
	dmat* extra=NULL;
	psd=psd2d(&extra, screen, 1./64.);
	out[2]=sqrt(psd_inte2(psd))*1e9;
	out[0]=sqrt(dsumsq(screen)/PN(screen))*1e9;
	out[3]=P(extra, 0);
	out[4]=P(extra, 1);
	dfree(extra);
	dfree(psd);
	dmat* st=stfun_batch(screen, NULL);
	out[5]=dsum(st)*1e9;
	out[6]=dmax(st)*1e13;
	dfree(st);
	dfree(screen);
}

/* Turbulence for the full-frame CPU path: nlayer screens kept as map_t. */
static map_t** g_atm=NULL;
static int g_natm=0;
void oref_atm_set(int nlayer, const double* const* screens, const long* nx, const long* ny, const double* dx,
	const double* ox, const double* oy, const double* ht, const double* vx, const double* vy){
	for(int i=0; i<g_natm; i++) mapfree(g_atm[i]);
	free(g_atm);
	g_natm=nlayer;
	g_atm=mycalloc(nlayer, map_t*);
	for(int i=0; i<nlayer; i++){
		map_t* m=g_atm[i]=mapnew(nx[i], ny[i], dx[i], dx[i]);
		memcpy(P(m), screens[i], sizeof(double)*nx[i]*ny[i]);
		m->ox=ox[i]; m->oy=oy[i]; m->ht=ht[i]; m->vx=vx[i]; m->vy=vy[i];
	}
}
map_t** oref_atm(int* nlayer){ *nlayer=g_natm; return g_atm; }

/* Closed-loop and static terms of the full frame's OPD (maos/wfsgrad.c:200-262
   and 373-377): mirror grids subtracted with prop (wrap=0, alpha=-1, as
   maos/sim_utils.c:1034-1052 sets up wfs_propdata_dm), loc_add_ptt,
   loc_add_focus (telescope) and loc_add_focus_offset (LLT zoom), the NCPA
   surface (powfs.opdadd) and the uplink tip/tilt on the LLT OPD.  ndm = 0 and
   zeros remove them. */
static map_t** g_dm=NULL;
static int g_ndm=0;
static int g_cl_use_dm=0;
static real g_cl_ptt[3]={0,0,0}, g_cl_focus_tel=0, g_cl_focus_llt=0, g_cl_lltptt[3]={0,0,0};
static dmat* g_cl_opdadd=NULL;
void oref_cl_set(int ndm, const double* const* surf, const long* nx, const long* ny, const double* dx,
	const double* ox, const double* oy, const double* ht, int use_dm, const double* ptt, double focus_tel,
	double focus_llt, const double* lltptt, const double* opdadd){
	for(int i=0; i<g_ndm; i++) mapfree(g_dm[i]);
	free(g_dm);
	g_ndm=ndm;
	g_dm=ndm?mycalloc(ndm, map_t*):NULL;
	for(int i=0; i<ndm; i++){
		map_t* m=g_dm[i]=mapnew(nx[i], ny[i], dx[i], dx[i]);
		memcpy(P(m), surf[i], sizeof(double)*nx[i]*ny[i]);
		m->ox=ox[i]; m->oy=oy[i]; m->ht=ht[i];
	}
	g_cl_use_dm=use_dm;
	for(int k=0; k<3; k++) g_cl_ptt[k]=ptt?ptt[k]:0;
	g_cl_focus_tel=focus_tel;
	g_cl_focus_llt=focus_llt;
	g_cl_lltptt[0]=0;
	g_cl_lltptt[1]=lltptt?lltptt[0]:0;
	g_cl_lltptt[2]=lltptt?lltptt[1]:0;
	dfree(g_cl_opdadd);
	g_cl_opdadd=NULL;
	if(opdadd){
		const long n=g_powfs[0].saloc->nloc*g_powfs[0].pts->nxsa*g_powfs[0].pts->nxsa;
		g_cl_opdadd=dnew(n, 1);
		memcpy(P(g_cl_opdadd), opdadd, sizeof(double)*n);
	}
}
static void cl_apply(dmat* opd, int iwfs){
	const parms_t* parms=g_parms;
	powfs_t* powfs=g_powfs;
	const real hs=parms->wfs[iwfs].hs;
	if(g_cl_focus_tel) loc_add_focus(opd, powfs[0].loc, g_cl_focus_tel);
	if(g_cl_focus_llt) loc_add_focus_offset(opd, powfs[0].loc, g_cl_focus_llt,
		P(parms->powfs[0].llt->ox, 0), P(parms->powfs[0].llt->oy, 0));
	if(g_cl_opdadd) dadd(&opd, 1, g_cl_opdadd, 1);
	if(g_cl_use_dm){
		for(int idm=0; idm<g_ndm; idm++){
			prop(&(propdata_t){.mapin=g_dm[idm], .ptsout=powfs[0].pts, .phiout=P(opd), .alpha=-1,
				.hs=hs, .thetax=parms->wfs[iwfs].thetax, .thetay=parms->wfs[iwfs].thetay, .wrap=0});
		}
	}
	if(g_cl_ptt[0]||g_cl_ptt[1]||g_cl_ptt[2]) loc_add_ptt(opd, g_cl_ptt, powfs[0].loc);
}

/* One complete WFS frame of the reference CPU path at step isim, as
   wfsgrad_iwfs runs it (maos/wfsgrad.c:170-194, 330-473): the ray trace of
   every layer split over 8 threads (LGS) or 2 (NGS) per layer
   (maos/sim_utils.c:1031), the LLT OPD for LGS, wfsints over
   thread_prep(0,nsa,NTHREAD), addnoise and shwfs_grad.  Returns seconds. */
double oref_frame_full_mt(int iwfs, int isim, double dt, double* ints, double* grad, unsigned int seed, int noisy){
	const parms_t* parms=g_parms;
	powfs_t* powfs=g_powfs;
	const long nsa=powfs[0].saloc->nloc;
	const long nopd=powfs[0].pts->nxsa;
	const real hs=parms->wfs[iwfs].hs;
	double t0=omp_get_wtime();
	dmat* opd=dnew(nsa*nopd*nopd, 1);
	const int nth=isinf(hs)?2:8;
	for(int ips=0; ips<g_natm; ips++){
		propdata_t pd={0};
		pd.mapin=g_atm[ips];
		pd.ptsout=powfs[0].pts;
		pd.phiout=P(opd);
		pd.alpha=1;
		pd.hs=hs;
		pd.thetax=parms->wfs[iwfs].thetax;
		pd.thetay=parms->wfs[iwfs].thetay;
		pd.shiftx=-g_atm[ips]->vx*dt*isim;
		pd.shifty=-g_atm[ips]->vy*dt*isim;
		pd.wrap=1;
		thread_t* thd=thread_prep(0, nsa, nth, prop_thread, &pd);
		CALL_THREAD(thd, 1);
		free(thd);
	}
	cl_apply(opd, iwfs);
	dmat* lltopd=NULL;
	if(powfs[0].llt){
		lltopd=dnew(powfs[0].llt->pts->nxsa, powfs[0].llt->pts->nysa);
		const real ox=P(parms->powfs[0].llt->ox, 0);
		const real oy=P(parms->powfs[0].llt->oy, 0);
		for(int ips=0; ips<g_natm; ips++){
			const real scale=1.-g_atm[ips]->ht/hs;
			if(scale<0) continue;
			prop(&(propdata_t){.mapin=g_atm[ips], .ptsout=powfs[0].llt->pts, .phiout=P(lltopd), .alpha=1,
				.hs=hs, .thetax=parms->wfs[iwfs].thetax-ox/hs, .thetay=parms->wfs[iwfs].thetay-oy/hs,
				.shiftx=ox-g_atm[ips]->vx*isim*dt, .shifty=oy-g_atm[ips]->vy*isim*dt, .wrap=1});
		}
		if(g_cl_lltptt[1]||g_cl_lltptt[2]) loc_add_ptt(lltopd, g_cl_lltptt, powfs[0].llt->loc);
	}
	double t1=omp_get_wtime();
	g_frame_isim=isim;
	double t=oref_frame_mt(iwfs, P(opd), lltopd?P(lltopd):NULL, ints, grad, seed, noisy);
	g_frame_isim=0;
	dfree(opd);
	dfree(lltopd);
	return (t1-t0)+t;
}

/* The OPD (nsa*nopd^2) and LLT OPD (llt_nx^2, if any) of WFS iwfs at step isim
   as oref_frame_full_mt forms them, closed-loop terms included. */
void oref_frame_opd(int iwfs, int isim, double dt, double* opdout, double* lltout){
	const parms_t* parms=g_parms;
	powfs_t* powfs=g_powfs;
	const long nsa=powfs[0].saloc->nloc;
	const long nopd=powfs[0].pts->nxsa;
	const real hs=parms->wfs[iwfs].hs;
	dmat* opd=dnew_do(nsa*nopd*nopd, 1, opdout, 0);
	dzero(opd);
	for(int ips=0; ips<g_natm; ips++){
		prop(&(propdata_t){.mapin=g_atm[ips], .ptsout=powfs[0].pts, .phiout=P(opd), .alpha=1, .hs=hs,
			.thetax=parms->wfs[iwfs].thetax, .thetay=parms->wfs[iwfs].thetay,
			.shiftx=-g_atm[ips]->vx*dt*isim, .shifty=-g_atm[ips]->vy*dt*isim, .wrap=1});
	}
	cl_apply(opd, iwfs);
	dfree(opd);
	if(lltout && powfs[0].llt){
		dmat* lltopd=dnew_do(powfs[0].llt->pts->nxsa, powfs[0].llt->pts->nysa, lltout, 0);
		dzero(lltopd);
		const real ox=P(parms->powfs[0].llt->ox, 0);
		const real oy=P(parms->powfs[0].llt->oy, 0);
		for(int ips=0; ips<g_natm; ips++){
			const real scale=1.-g_atm[ips]->ht/hs;
			if(scale<0) continue;
			prop(&(propdata_t){.mapin=g_atm[ips], .ptsout=powfs[0].llt->pts, .phiout=P(lltopd), .alpha=1,
				.hs=hs, .thetax=parms->wfs[iwfs].thetax-ox/hs, .thetay=parms->wfs[iwfs].thetay-oy/hs,
				.shiftx=ox-g_atm[ips]->vx*isim*dt, .shifty=oy-g_atm[ips]->vy*isim*dt, .wrap=1});
		}
		if(g_cl_lltptt[1]||g_cl_lltptt[2]) loc_add_ptt(lltopd, g_cl_lltptt, powfs[0].llt->loc);
		dfree(lltopd);
	}
}

/* The second ETF of the time interpolation: the reference's own
   setup_shwfs_etf in mode 2 (maos/powfs.c:1157-1175) for the sodium layer
   focused at hs + deltah, and the interpolation period coldtrat
   (maos/wfsints.c:215-223). */
void oref_setup_etf2(double deltah, int coldtrat){
	setup_shwfs_etf(g_powfs, g_parms, 0, 2, 0, deltah, 0);
	g_parms->powfs[0].llt->coldtrat=coldtrat;
}
void oref_get_etf2(int isa, double* out){
	cmat* e=P(g_powfs[0].etfsim2[0].etf, isa, 0);
	copy_vec(out, (double*)P(e), 2*PN(e));
}

/* Geometric z-tilt gradients (2*nsa) of an OPD (nsa*nopd^2) over the
   powfs's subapertures: the reference's pts_mcc_ptt and dcellinvspd_each
   (maos/powfs.c:633-645) and pts_ztilt (math/loc.c:839-885). */
void oref_ztilt(const double* opd, double* grad){
	const long nsa=g_powfs[0].saloc->nloc;
	const double* amp=P(P(g_powfs[0].amp, 0));
	dcell* mcc=pts_mcc_ptt(g_powfs[0].pts, amp);
	dcell* imcc=dcellinvspd_each(mcc);
	dmat* g=dnew(2*nsa, 1);
	pts_ztilt(&g, g_powfs[0].pts, imcc, amp, opd);
	copy_vec(grad, P(g), 2*nsa);
	dfree(g);
	dcellfree(imcc);
	dcellfree(mcc);
}

/* The G-tilt operator GS0 of the powfs as maos/powfs.c:619-626 makes it:
   mkg (lib/mkg.c:471) on the WFS OPD grid with the amplitude, subaperture
   list, saa and saat; CSC export and GS0*opd by the reference's dspmm. */
static void gs0_make(void){
	if(g_gs0) return;
	g_gs0=mkg(g_powfs[0].loc, g_powfs[0].loc, P(g_powfs[0].amp, 0), g_powfs[0].saloc, P(g_powfs[0].saa, 0),
		g_parms->powfs[0].saat, 1, 0, 0, 1);
}
long oref_gs0_nnz(void){ gs0_make(); return (long)g_gs0->pp[g_gs0->ny]; }
void oref_get_gs0(long* nrow, long* ncol, int* pp, int* pi, double* px){
	gs0_make();
	*nrow=g_gs0->nx;
	*ncol=g_gs0->ny;
	const long nnz=g_gs0->pp[g_gs0->ny];
	for(long i=0; i<=g_gs0->ny; i++) pp[i]=(int)g_gs0->pp[i];
	for(long i=0; i<nnz; i++){ pi[i]=(int)g_gs0->pi[i]; px[i]=g_gs0->px[i]; }
}
void oref_gtilt(const double* opd, double* grad){
	gs0_make();
	dmat* o=dnew_do(g_gs0->ny, 1, (double*)opd, 0);
	dmat* g=dnew(g_gs0->nx, 1);
	dspmm(&g, g_gs0, o, "nn", 1);
	copy_vec(grad, P(g), g_gs0->nx);
	dfree(g);
	dfree(o);
}

/* The reference's own .bin writer and reader (writebin, math/cell.c:330-337;
   dread/readbin, math/cell.c:545-559) on plain arrays, to check the
   product's format code byte for byte and to write golden fixtures. */
void oref_writebin_d(const char* fn, const double* p, long nx, long ny, const char* keywords){
	dmat* a=dnew(nx, ny);
	copy_vec(P(a), p, nx*ny);
	if(keywords) a->keywords=strdup(keywords);
	writebin(a, "%s", fn);
	dfree(a);
}
void oref_writebin_f(const char* fn, const float* p, long nx, long ny, const char* keywords){
	smat* a=snew(nx, ny);
	memcpy(P(a), p, sizeof(float)*nx*ny);
	if(keywords) a->keywords=strdup(keywords);
	writebin(a, "%s", fn);
	sfree(a);
}
void oref_writebin_c(const char* fn, const double* p, long nx, long ny){
	cmat* a=cnew(nx, ny);
	memcpy(P(a), p, sizeof(double)*2*nx*ny);
	writebin(a, "%s", fn);
	cfree(a);
}
/* A cell of n members, member i of nx[i] x ny[i] doubles (0 x 0 = empty). */
void oref_writebin_dcell(const char* fn, int n, const long* nx, const long* ny, const double* const* p,
	const char* keywords){
	dcell* c=dcellnew(n, 1);
	for(int i=0; i<n; i++){
		if(nx[i]*ny[i]>0){
			P(c, i)=dnew(nx[i], ny[i]);
			copy_vec(P(P(c, i)), p[i], nx[i]*ny[i]);
		}
	}
	if(keywords) c->keywords=strdup(keywords);
	writebin(c, "%s", fn);
	dcellfree(c);
}
void oref_writebin_gs0(const char* fn){
	gs0_make();
	writebin(g_gs0, "%s", fn);
}
/* dread of a file: returns nx*ny (copied up to nmax), dimensions in *nx, *ny. */
long oref_readbin_d(const char* fn, double* out, long nmax, long* nx, long* ny){
	dmat* a=dread("%s", fn);
	if(!a){ *nx=*ny=0; return 0; }
	*nx=a->nx; *ny=a->ny;
	long n=a->nx*a->ny;
	copy_vec(out, P(a), n<nmax?n:nmax);
	dfree(a);
	return n;
}

/* Science aperture and open-loop evaluation by the reference's own code:
   setup_aper (maos/aper.c:32-150) for an annulus (no loaded locs, amplitude
   map, pupil mask or distortion), then per frame the atmosphere traced onto
   aper->locs as perfevl_ievl does (prop with the locs' column statistics,
   maos/sim_utils.c:729-743 and maos/perfevl.c:146-166), loc_calc_ptt
   (math/loc.c:653-709) and, for the PSF, loc_sub_ptt when pttr and
   locfft_psf followed by |.|^2 (maos/perfevl.c:206-226). */
static loc_t* g_elocs=NULL;
static dmat* g_eamp=NULL;
static dmat* g_emcc=NULL;
static dmat* g_eimcc=NULL;
static real g_eipcc=0;
static locfft_t* g_elocfft=NULL;
long oref_evl_setup(double D, double Din, double dx, int nwvl, const double* wvl, const long* nembed){
	if(g_elocfft){ locfft_free(g_elocfft); g_elocfft=NULL; }
	locfree(g_elocs); dfree(g_eamp); dfree(g_emcc); dfree(g_eimcc);
	map_t* smap=NULL;
	create_metapupil(&smap, 0, 0, NULL, D, 0, dx, dx, 0, dx, 0, 0, 0, 0);
	g_elocs=loc_from_map(smap, 0);
	mapfree(smap);
	g_eamp=mkamp(g_elocs, NULL, 0, 0, D, Din);
	loc_reduce(g_elocs, g_eamp, EPS, 1, NULL);
	loc_create_stat(g_elocs);
	dnormalize_sum(g_eamp, 1);
	g_emcc=loc_mcc_ptt(g_elocs, P(g_eamp));
	g_eipcc=1./P(g_emcc, 0);
	g_eimcc=dinvspd(g_emcc);
	if(nwvl>0){
		dmat* w=dnew(nwvl, 1);
		lmat* fs=lnew(nwvl, 1);
		for(int i=0; i<nwvl; i++){ P(w, i)=wvl[i]; P(fs, i)=nembed[i]; }
		g_elocfft=locfft_init(g_elocs, g_eamp, w, fs, 2, 0);
		dfree(w);
		lfree(fs);
	}
	return g_elocs->nloc;
}
/* The aperture built by oref_evl_setup, for the adapter driver (adapter_driver.c). */
void oref_evl_aper(loc_t** locs, dmat** amp, locfft_t** locfft){
	*locs=g_elocs; *amp=g_eamp; *locfft=g_elocfft;
}
void oref_evl_get_aper(double* locx, double* locy, double* amp){
	copy_vec(locx, g_elocs->locx, g_elocs->nloc);
	copy_vec(locy, g_elocs->locy, g_elocs->nloc);
	copy_vec(amp, P(g_eamp), g_elocs->nloc);
}
/* One frame of direction (thetax, thetay, hs): opd (nloc), wfe {PR, TT,
   PTTR}, coeff {p, tip, tilt}, and per wavelength the psfsize^2 |PSF|^2
   (column-major, concatenated), when psf is not NULL. */
void oref_evl_frame(double thetax, double thetay, double hs, int isim, double dt, int pttr, int nwvl,
	const long* psfsize, double* opd, double* wfe, double* coeff, double* psf){
	dmat* o=dnew(g_elocs->nloc, 1);
	for(int ips=0; ips<g_natm; ips++){
		prop(&(propdata_t){.mapin=g_atm[ips], .ostat=g_elocs->stat, .phiout=P(o), .alpha=1, .hs=hs,
			.thetax=thetax, .thetay=thetay, .shiftx=-g_atm[ips]->vx*isim*dt, .shifty=-g_atm[ips]->vy*isim*dt,
			.wrap=1});
	}
	copy_vec(opd, P(o), g_elocs->nloc);
	loc_calc_ptt(wfe, coeff, g_elocs, g_eipcc, g_eimcc, P(g_eamp), P(o));
	if(psf && g_elocfft){
		if(pttr) loc_sub_ptt(o, coeff, g_elocs);
		lmat* ps=lnew(nwvl, 1);
		for(int i=0; i<nwvl; i++) P(ps, i)=psfsize[i];
		ccell* psf2s=NULL;
		locfft_psf(&psf2s, g_elocfft, o, ps, 0);
		long off=0;
		for(int i=0; i<nwvl; i++){
			cmat* c=P(psf2s, i);
			for(long k=0; k<PN(c); k++) psf[off+k]=creal(P(c, k)*conj(P(c, k)));
			off+=PN(c);
		}
		ccellfree(psf2s);
		lfree(ps);
	}
	dfree(o);
}
