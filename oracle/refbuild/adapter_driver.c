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
		memcpy(grad+(iwfs-iwfs0)*ng, P(P(g_sim->gradcl, iwfs)), sizeof(double)*ng);
	}
	return 0;
}
