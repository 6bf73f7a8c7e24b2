/*
 * Test driver of the MAOS-side adapter (maos_b200/csrc/adapter/wfs_b200.c). Test infrastructure.
 *
 * It calls MAOS's GPU wavefront-sensor seam in the order the simulator does: gpu_wfsgrad_init
 * at setup (maos/setup.c:192-203), gpu_atm2gpu for the screens (maos/sim.c:79), then per frame
 * gpu_wfsgrad_queue with a thread_t over the WFS range (maos/sim_utils.c:1497-1504) and
 * gpu_wfsgrad_sync into simu->gradcl (maos/wfsgrad.c:834-838). The parms_t, powfs_t and
 * turbulence are the ones the reference's own setup built in ref_driver.c (oref_setup,
 * oref_atm_set), so every array reaches the library the way the adapter reads it from MAOS.
 */
#include <string.h>
#include "gpu_sim.h"

parms_t* oref_parms(void);
powfs_t* oref_powfs(void);
map_t** oref_atm(int* nlayer);
void oref_evl_aper(loc_t** locs, dmat** amp, locfft_t** locfft);

static sim_t* g_sim=NULL;

/* Setup through the seam; noisy sets powfs.noisy, dt sets sim.dt. Returns the number of WFS. */
int oadp_init(int noisy, double dt){
	parms_t* parms=oref_parms();
	powfs_t* powfs=oref_powfs();
	if(!parms || !powfs) return -1;
	parms->powfs[0].noisy=noisy;
	parms->sim.dt=dt;
	gpu_wfsgrad_init(parms, powfs);
	int n=0;
	map_t** atm=oref_atm(&n);
	mapcell* ac=mapcellnew(n, 1);
	for(int i=0; i<n; i++) P(ac, i)=mapref(atm[i]);
	gpu_atm2gpu(ac, NULL, parms, 0, 0);
	cellfree(ac);
	if(g_sim){
		dcellfree(g_sim->gradcl);
		free(g_sim);
	}
	g_sim=mycalloc(1, sim_t);
	g_sim->parms=parms;
	g_sim->powfs=powfs;
	g_sim->save=mycalloc(1, sim_save_t);
	parms->sim.closeloop=0;
	g_sim->gradcl=dcellnew(parms->nwfs, 1);
	return parms->nwfs;
}

/* New ETF pair of powfs 0 through gpu_wfsgrad_update_etf, as sim_update_etf does
   (maos/sim_utils.c:338) after the reference's setup made etfsim2 (oref_setup_etf2). */
void oadp_update_etf(void){
	gpu_wfsgrad_update_etf(oref_parms(), oref_powfs(), 0);
}

/* Seeds the noise of every WFS through gpu_wfsgrad_seeding from a reference MT19937 stream. */
void oadp_seed(unsigned int seed){
	rand_t rs;
	seed_rand(&rs, seed);
	gpu_wfsgrad_seeding(oref_parms(), oref_powfs(), &rs);
}

/* Frame isim of WFS iwfs0..iwfs1-1: queue, then sync each; grad receives (iwfs1-iwfs0) blocks
   of 2*nsa gradients (x then y). */
int oadp_frame(int isim, int iwfs0, int iwfs1, double* grad){
	if(!g_sim) return -1;
	const long ng=2*g_sim->powfs[0].saloc->nloc;
	g_sim->wfsisim=isim;
	thread_t t={0};
	t.start=iwfs0;
	t.end=iwfs1;
	t.nthread=1;
	t.data=g_sim;
	gpu_wfsgrad_queue(&t);
	for(int iwfs=iwfs0; iwfs<iwfs1; iwfs++){
		gpu_wfsgrad_sync(g_sim, iwfs);
		const dmat* g=P(g_sim->gradcl, iwfs);  /* still NULL before the WFS's first output */
		if(g) memcpy(grad+(iwfs-iwfs0)*ng, P(g), sizeof(double)*ng);
		else memset(grad+(iwfs-iwfs0)*ng, 0, sizeof(double)*ng);
	}
	return 0;
}

/* Closed-loop state of the simulation as the adapter reads it from sim_t: the DM surfaces
   (simu->dmrealsq, uploaded through gpu_dmreal2gpu as maos/filter.c:561 does), the tip/tilt
   mirror (simu->ttmreal), the per-WFS FSM (simu->fsmreal: downlink for NGS, uplink for LGS),
   the telescope focus (simu->telfocusreal) and the LGS trombone (simu->zoomint, one per WFS).
   closeloop sets parms->sim.closeloop. */
int oadp_set_cl(int closeloop, int ndm, const double* const* surf, const long* nx, const long* ny, const double* dx,
	const double* ox, const double* oy, const double* ht, const double* ttm, const double* fsm, double telfocus,
	const double* zoomint){
	sim_t* simu=g_sim;
	if(!simu) return -1;
	parms_t* parms=(parms_t*)simu->parms;
	parms->sim.closeloop=closeloop;
	cellfree(simu->dmrealsq);
	simu->dmrealsq=NULL;
	if(ndm){
		simu->dmrealsq=mapcellnew(ndm, 1);
		for(int i=0; i<ndm; i++){
			map_t* m=P(simu->dmrealsq, i)=mapnew(nx[i], ny[i], dx[i], dx[i]);
			memcpy(P(m), surf[i], sizeof(double)*nx[i]*ny[i]);
			m->ox=ox[i]; m->oy=oy[i]; m->ht=ht[i];
		}
	}
	dfree(simu->ttmreal);
	simu->ttmreal=NULL;
	if(ttm){ simu->ttmreal=dnew(2, 1); P(simu->ttmreal, 0)=ttm[0]; P(simu->ttmreal, 1)=ttm[1]; }
	dcellfree(simu->fsmreal);
	simu->fsmreal=NULL;
	if(fsm){
		simu->fsmreal=dcellnew(parms->nwfs, 1);
		for(int i=0; i<parms->nwfs; i++){
			P(simu->fsmreal, i)=dnew(2, 1);
			P(P(simu->fsmreal, i), 0)=fsm[2*i];
			P(P(simu->fsmreal, i), 1)=fsm[2*i+1];
		}
	}
	dcellfree(simu->telfocusreal);
	simu->telfocusreal=NULL;
	if(telfocus!=0){ simu->telfocusreal=dcellnew(1, 1); P(simu->telfocusreal, 0)=dnew(1, 1); P(P(simu->telfocusreal, 0), 0)=telfocus; }
	dfree(simu->zoomint);
	simu->zoomint=NULL;
	if(zoomint){ simu->zoomint=dnew(parms->nwfs, 1); for(int i=0; i<parms->nwfs; i++) P(simu->zoomint, i)=zoomint[i]; }
	if(simu->dmrealsq) gpu_dmreal2gpu(simu->dmrealsq);
	return 0;
}

/* The NCPA surface of every WFS of powfs 0 (powfs.opdadd, nsa*nopd^2 values, the same for all WFS)
   through gpu_wfssurf2gpu, as maos/setup.c:202 does; NULL removes it. */
int oadp_set_opdadd(const double* opd){
	parms_t* parms=oref_parms();
	powfs_t* powfs=oref_powfs();
	dcellfree(powfs[0].opdadd);
	powfs[0].opdadd=NULL;
	if(opd){
		const long n=powfs[0].saloc->nloc*powfs[0].pts->nxsa*powfs[0].pts->nxsa;
		powfs[0].opdadd=dcellnew(parms->powfs[0].nwfs, 1);
		for(int i=0; i<parms->powfs[0].nwfs; i++){
			P(powfs[0].opdadd, i)=dnew(n, 1);
			memcpy(P(P(powfs[0].opdadd, i)), opd, sizeof(double)*n);
		}
	}
	gpu_wfssurf2gpu(parms, powfs);
	return 0;
}

/* Sets one option of the reference's parms_t/powfs_t (powfs 0) before oadp_init, for the tests of
   the options the adapter serves or refuses:
     1 powfs.nwvl   2 llt.nhs   3 one amplitude map per WFS   4 powfs.phytype_sim   5 powfs.moao
     6 powfs.fieldstop   7 powfs.dither   8 powfs.pistatout   9 sim.idealwfs   10 a cubic DM (dm.iac)
     11 atm.dtrat   12 powfs.type   13 powfs.usephy   14 powfs.gtype_sim   15 powfs.phystep
     16 powfs.step   17 powfs.dtrat */
int oadp_poke(int what, double v){
	parms_t* parms=oref_parms();
	powfs_t* powfs=oref_powfs();
	if(!parms || !powfs) return -1;
	powfs_cfg_t* pc=&parms->powfs[0];
	switch(what){
	case 1: pc->nwvl=(int)v; break;
	case 2: if(!pc->llt) return -1; pc->llt->nhs=(int)v; break;
	case 3:{
		dcell* a=dcellnew(2, 1);
		P(a, 0)=dref(P(powfs[0].amp, 0));
		P(a, 1)=dref(P(powfs[0].amp, 0));
		dcellfree(powfs[0].amp);
		powfs[0].amp=a;
		break;
	}
	case 4: pc->phytype_sim=(int)v; break;
	case 5: pc->moao=(int)v; break;
	case 6: pc->fieldstop=v; break;
	case 7: pc->dither=(int)v; break;
	case 8: pc->pistatout=(int)v; break;
	case 9: parms->sim.idealwfs=(int)v; break;
	case 10:
		parms->ndm=1;
		parms->dm=mycalloc(1, dm_cfg_t);
		parms->dm[0].iac=v;
		break;
	case 11: parms->atm.dtrat=(int)v; break;
	case 12: pc->type=(int)v; break;
	case 13: pc->usephy=(int)v; break;
	case 14: pc->gtype_sim=(int)v; break;
	case 15: pc->phystep=(int)v; break;
	case 16: pc->step=(int)v; break;
	case 17: pc->dtrat=(int)v; break;
	default: return -1;
	}
	return 0;
}

/* ---- science path (gpu_perfevl_*), on the aperture of oref_evl_setup ---- */
static parms_t* g_eparms=NULL;
static aper_t* g_eaper=NULL;
static sim_t* g_esim=NULL;

static dmat* dvec(int n, const double* v){
	dmat* d=dnew(n, 1);
	for(int i=0; i<n; i++) P(d, i)=v[i];
	return d;
}

/* Setup as maos/setup.c does it for an open-loop run with nsim frames: gpu_perfevl_init,
   gpu_atm2gpu, gpu_perfevl_init_sim. psfsize per wavelength; pttr for every direction. */
int oadp_evl_init(int nevl, const double* thetax, const double* thetay, const double* hs, int nwvl,
	const double* wvl, const long* psfsize, int pttr, double dt, int nsim){
	parms_t* parms=g_eparms=mycalloc(1, parms_t);
	parms->evl.nevl=nevl;
	parms->evl.thetax=dvec(nevl, thetax);
	parms->evl.thetay=dvec(nevl, thetay);
	parms->evl.hs=dvec(nevl, hs);
	parms->evl.nwvl=nwvl;
	parms->evl.wvl=dvec(nwvl, wvl);
	parms->evl.psfsize=lnew(nwvl, 1);
	for(int i=0; i<nwvl; i++) P(parms->evl.psfsize, i)=psfsize[i];
	parms->evl.pttr=lnew(nevl, 1);
	for(int i=0; i<nevl; i++) P(parms->evl.pttr, i)=pttr;
	parms->evl.nmod=3;
	parms->evl.psfmean=nwvl>0;
	parms->evl.psfisim=0;
	parms->sim.dt=dt;
	aper_t* aper=g_eaper=mycalloc(1, aper_t);
	oref_evl_aper(&aper->locs, &aper->amp, &aper->locfft);
	gpu_perfevl_init(parms, aper);
	int n=0;
	map_t** atm=oref_atm(&n);
	mapcell* ac=mapcellnew(n, 1);
	for(int i=0; i<n; i++) P(ac, i)=mapref(atm[i]);
	gpu_atm2gpu(ac, NULL, parms, 0, 0);
	cellfree(ac);
	gpu_perfevl_init_sim(parms, aper);
	sim_t* simu=g_esim=mycalloc(1, sim_t);
	simu->parms=parms;
	simu->aper=aper;
	simu->olep=dcellnew(nevl, 1);
	simu->olmp=dcellnew(nevl, 1);
	for(int i=0; i<nevl; i++){
		P(simu->olep, i)=dnew(3, nsim);
		P(simu->olmp, i)=dnew(3, nsim);
	}
	return nevl;
}

/* Frame isim of every direction, queued and synced over two "threads" as the simulator splits
   the directions; wfe and coeff receive nevl x 3 from simu->olep and simu->olmp. */
int oadp_evl_frame(int isim, double* wfe, double* coeff){
	sim_t* simu=g_esim;
	if(!simu) return -1;
	const int nevl=simu->parms->evl.nevl;
	simu->perfisim=isim;
	const long half=nevl/2;
	thread_t t[2]={{0}, {0}};
	t[0].start=0; t[0].end=half; t[0].data=simu;
	t[1].start=half; t[1].end=nevl; t[1].data=simu;
	gpu_perfevl_queue(&t[0]);
	gpu_perfevl_queue(&t[1]);
	gpu_perfevl_sync(&t[1]);
	gpu_perfevl_sync(&t[0]);
	for(int i=0; i<nevl; i++){
		memcpy(wfe+3*i, PCOL(P(simu->olep, i), isim), sizeof(double)*3);
		memcpy(coeff+3*i, PCOL(P(simu->olmp, i), isim), sizeof(double)*3);
	}
	return 0;
}
