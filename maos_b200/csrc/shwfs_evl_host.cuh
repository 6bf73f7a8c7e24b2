// Science-path evaluation: host side of include/shwfs_evl.h.  Included at the
// end of shwfs_api.cu, whose context, buffers and ray-trace helpers it uses.
#pragma once
#include "../../include/shwfs_evl.h"
#include "shwfs_evl.cuh"

struct EvlPsf {
	int N = 0, psfsize = 0, h = 0, offx = 0, offy = 0;
	double wvl = 0;
	DevBuf<float2> tw;   // exp(-2 pi i k / N), k < N
	DevBuf<float> psf;   // nevl * psfsize^2 sums, crop column major
};

struct EvlState {
	long nloc = 0;
	double dx = 0, ox = 0, oy = 0;
	int nX = 0, nY = 0, ntx = 0, nty = 0, nslot = 0;
	DevBuf<double> torigx, torigy;  // tile origins, by slot
	DevBuf<int> tile_slot, slot_tile, loc_addr;
	DevBuf<float> amp;              // nslot*256
	double ipcc = 0, imcc[9] = {0};
	DevBuf<double> imcc_d;
	struct Dir {
		double thetax, thetay, hs;
	};
	std::vector<Dir> dirs;
	DevBuf<float> opd;              // nevl * nslot * 256
	DevBuf<double> sums, coeff;     // nevl*4, nevl*3
	double* sums_h = nullptr;       // pinned nevl*4
	size_t sums_h_n = 0;
	std::vector<EvlPsf> psf;
	int pttr = 0;
	long nframe = 0;
	DevBuf<float2> T;
	int queued = 0;
};

static void evl_free(shwfs_ctx* ctx) {
	EvlState* E = ctx->evl;
	if (!E) return;
	E->torigx.free_();
	E->torigy.free_();
	E->tile_slot.free_();
	E->slot_tile.free_();
	E->loc_addr.free_();
	E->amp.free_();
	E->imcc_d.free_();
	E->opd.free_();
	E->sums.free_();
	E->coeff.free_();
	E->T.free_();
	for (auto& p : E->psf) {
		p.tw.free_();
		p.psf.free_();
	}
	if (E->sums_h) cudaFreeHost(E->sums_h);
	delete E;
	ctx->evl = nullptr;
}

static EvlRaster evl_raster(const EvlState& E) {
	EvlRaster R;
	R.nslot = E.nslot;
	R.ntx = E.ntx;
	R.nty = E.nty;
	R.nX = E.nX;
	R.nY = E.nY;
	R.ox = E.ox;
	R.oy = E.oy;
	R.dx = E.dx;
	R.tile_slot = E.tile_slot.p;
	R.slot_tile = E.slot_tile.p;
	R.amp = E.amp.p;
	return R;
}

// Inverse of the symmetric 3x3 moment matrix (dinvspd on aper->mcc, maos/aper.c:111-113).
static bool inv3_sym(const double m[9], double out[9]) {
	const double a00 = m[0], a01 = m[3], a02 = m[6], a11 = m[4], a12 = m[7], a22 = m[8];
	const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
	const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
	const double det = a00 * c00 + a01 * c01 + a02 * c02;
	if (!(det > 0) || !isfinite(det)) return false;
	const double c[9] = {c00, c01, c02, c01, c11, c12, c02, c12, c22};
	for (int i = 0; i < 9; i++) out[i] = c[i] / det;
	return true;
}

extern "C" {

int shwfs_evl_set_aper(shwfs_ctx* ctx, long nloc, const double* locx, const double* locy, double dx,
	const double* amp) {
	if (!ctx || nloc <= 0 || !locx || !locy || !amp || !(dx > 0))
		return ctx ? fail(ctx, SHWFS_EINVAL, "evl_set_aper: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (!ctx->evl) ctx->evl = new EvlState();
	EvlState& E = *ctx->evl;
	double xmin = locx[0], ymin = locy[0], xmax = locx[0], ymax = locy[0];
	for (long i = 1; i < nloc; i++) {
		xmin = std::min(xmin, locx[i]);
		xmax = std::max(xmax, locx[i]);
		ymin = std::min(ymin, locy[i]);
		ymax = std::max(ymax, locy[i]);
	}
	const long nX = (long)llround((xmax - xmin) / dx) + 1, nY = (long)llround((ymax - ymin) / dx) + 1;
	if (nX > 65536 || nY > 65536) return fail(ctx, SHWFS_EINVAL, "evl_set_aper: aperture of %ldx%ld points too large", nX, nY);
	const int ntx = (int)((nX + 15) / 16), nty = (int)((nY + 15) / 16);
	std::vector<int> X(nloc), Y(nloc), tslot((size_t)ntx * nty, -1);
	std::vector<char> used((size_t)ntx * nty, 0);
	for (long i = 0; i < nloc; i++) {
		const double fx = (locx[i] - xmin) / dx, fy = (locy[i] - ymin) / dx;
		X[i] = (int)llround(fx);
		Y[i] = (int)llround(fy);
		if (fabs(fx - X[i]) > 1e-6 || fabs(fy - Y[i]) > 1e-6)
			return fail(ctx, SHWFS_EINVAL, "evl_set_aper: point %ld is off the grid of spacing %g", i, dx);
		used[(size_t)(Y[i] >> 4) * ntx + (X[i] >> 4)] = 1;
	}
	std::vector<int> stile;  // tiles holding aperture points, in raster order
	for (int t = 0; t < ntx * nty; t++)
		if (used[t]) {
			tslot[t] = (int)stile.size();
			stile.push_back(t);
		}
	const int nslot = (int)stile.size();
	std::vector<float> araster((size_t)nslot * 256, 0.f);
	std::vector<int> addr(nloc);
	std::vector<char> seen((size_t)nslot * 256, 0);
	double mcc[9] = {0};
	for (long i = 0; i < nloc; i++) {
		const int slot = tslot[(size_t)(Y[i] >> 4) * ntx + (X[i] >> 4)];
		const int a = slot * 256 + (Y[i] & 15) * 16 + (X[i] & 15);
		if (seen[a]) return fail(ctx, SHWFS_EINVAL, "evl_set_aper: point %ld repeats a grid point", i);
		seen[a] = 1;
		addr[i] = a;
		araster[a] = (float)amp[i];
		// loc_mcc_ptt (math/loc.c:612-650)
		const double b[3] = {1, locx[i], locy[i]};
		for (int p = 0; p < 3; p++)
			for (int q = 0; q < 3; q++) mcc[p + 3 * q] += amp[i] * b[p] * b[q];
	}
	double imcc[9];
	if (!inv3_sym(mcc, imcc)) return fail(ctx, SHWFS_EINVAL, "evl_set_aper: singular moment matrix (no amplitude?)");
	std::vector<double> tox(nslot), toy(nslot);
	for (int s = 0; s < nslot; s++) {
		tox[s] = xmin + 16.0 * (stile[s] % ntx) * dx;
		toy[s] = ymin + 16.0 * (stile[s] / ntx) * dx;
	}
	if ((r = dev_upload(ctx, E.torigx, tox.data(), tox.size())) || (r = dev_upload(ctx, E.torigy, toy.data(), toy.size())) ||
		(r = dev_upload(ctx, E.tile_slot, tslot.data(), tslot.size())) ||
		(r = dev_upload(ctx, E.slot_tile, stile.data(), stile.size())) ||
		(r = dev_upload(ctx, E.loc_addr, addr.data(), addr.size())) ||
		(r = dev_upload(ctx, E.amp, araster.data(), araster.size())) || (r = dev_upload(ctx, E.imcc_d, imcc, 9)))
		return r;
	E.nloc = nloc;
	E.dx = dx;
	E.ox = xmin;
	E.oy = ymin;
	E.nX = (int)nX;
	E.nY = (int)nY;
	E.ntx = ntx;
	E.nty = nty;
	E.nslot = nslot;
	E.ipcc = 1. / mcc[0];
	memcpy(E.imcc, imcc, sizeof(imcc));
	for (auto& p : E.psf) {  // the embedding depends on the aperture: set the PSF again
		p.tw.free_();
		p.psf.free_();
	}
	E.psf.clear();
	E.queued = 0;
	CK(cudaStreamSynchronize(ctx->stream));
	return 0;
}

int shwfs_evl_add_dir(shwfs_ctx* ctx, double thetax, double thetay, double hs, int* ievl) {
	if (!ctx || !ctx->evl || !ievl) return ctx ? fail(ctx, SHWFS_ESTATE, "evl_add_dir: set the aperture first") : SHWFS_EINVAL;
	EvlState& E = *ctx->evl;
	if ((int)E.dirs.size() >= 1024) return fail(ctx, SHWFS_EINVAL, "evl_add_dir: too many directions");
	E.dirs.push_back({thetax, thetay, hs});
	*ievl = (int)E.dirs.size() - 1;
	for (auto& p : E.psf) p.psf.free_();  // sized by the number of directions: zeroed again on next use
	E.queued = 0;
	return 0;
}

int shwfs_evl_set_psf(shwfs_ctx* ctx, int nwvl, const double* wvl, const int* nembed, const int* psfsize, int pttr) {
	if (!ctx || !ctx->evl || nwvl < 0 || nwvl > 16 || (nwvl && (!wvl || !nembed)))
		return ctx ? fail(ctx, SHWFS_EINVAL, "evl_set_psf: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	EvlState& E = *ctx->evl;
	std::vector<EvlPsf> v(nwvl);
	for (int w = 0; w < nwvl; w++) {
		const int N = nembed[w];
		if (N < 64 || N > 4096 || (N & (N - 1)))
			return fail(ctx, SHWFS_EINVAL, "evl_set_psf: nembed %d must be a power of two in [64, 4096]", N);
		const int ps = (psfsize && psfsize[w] > 0) ? psfsize[w] : N;
		if (ps > N || (ps & 1)) return fail(ctx, SHWFS_EINVAL, "evl_set_psf: psfsize %d must be even and <= nembed", ps);
		if (!(wvl[w] > 0)) return fail(ctx, SHWFS_EINVAL, "evl_set_psf: wavelength must be positive");
		// loc_create_embed (math/loc.c:147-179): point X of the aperture grid
		// lands at column X + (nembed - nX + 1) / 2
		const int offx = (N - E.nX + 1) / 2, offy = (N - E.nY + 1) / 2;
		if (offx < 0 || offy < 0 || E.nX - 1 + offx >= N || E.nY - 1 + offy >= N)
			return fail(ctx, SHWFS_EINVAL, "evl_set_psf: nembed %d smaller than the aperture (%dx%d points)", N, E.nX, E.nY);
		v[w].N = N;
		v[w].psfsize = ps;
		v[w].h = ps / 2;
		v[w].offx = offx;
		v[w].offy = offy;
		v[w].wvl = wvl[w];
		std::vector<float2> tw(N);
		for (int k = 0; k < N; k++) {
			const double a = -2.0 * M_PI * k / N;
			tw[k] = make_float2((float)cos(a), (float)sin(a));
		}
		if ((r = dev_upload(ctx, v[w].tw, tw.data(), tw.size()))) return r;
	}
	for (auto& p : E.psf) {
		p.tw.free_();
		p.psf.free_();
	}
	E.psf.swap(v);
	E.pttr = pttr ? 1 : 0;
	E.nframe = 0;
	return 0;
}

int shwfs_evl_psf_reset(shwfs_ctx* ctx) {
	if (!ctx || !ctx->evl) return ctx ? fail(ctx, SHWFS_ESTATE, "evl_psf_reset: no aperture") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	for (auto& p : ctx->evl->psf)
		if (p.psf.p) CK(cudaMemsetAsync(p.psf.p, 0, sizeof(float) * p.psf.n, ctx->stream));
	ctx->evl->nframe = 0;
	return 0;
}

}  // extern "C"

template <int N>
static int evl_launch_psf(shwfs_ctx* ctx, EvlState& E, EvlPsf& P, int nevl) {
	constexpr int R = 4096 / N;  // rows per block: 512 radix-8 groups, one per thread
	const size_t smem_r = (size_t)R * evl_row_len<N>() * sizeof(float2), smem_c = (size_t)evl_row_len<N>() * sizeof(float2);
	if (smem_r > 48 * 1024)
		CK(cudaFuncSetAttribute(evl_psf_rows_kernel<N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r));
	const EvlRaster Ra = evl_raster(E);
	const float twoinvwvl = (float)(2.0 / P.wvl);
	evl_psf_rows_kernel<N, R><<<dim3((E.nY + R - 1) / R, nevl), EVL_THREADS, smem_r, ctx->stream>>>(
		Ra, E.opd.p, E.coeff.p, E.pttr, twoinvwvl, P.offx, P.h, P.tw.p, E.T.p, E.nY);
	CK(cudaGetLastError());
	evl_psf_cols_kernel<N><<<dim3(2 * P.h, nevl), EVL_THREADS, smem_c, ctx->stream>>>(E.T.p, E.nY, E.nY, P.offy, P.h, P.tw.p,
		P.psf.p);
	CK(cudaGetLastError());
	return 0;
}

extern "C" {

int shwfs_evl_queue(shwfs_ctx* ctx, int isim, int do_psf) {
	if (!ctx || !ctx->evl || ctx->evl->dirs.empty())
		return ctx ? fail(ctx, SHWFS_ESTATE, "evl_queue: set the aperture and at least one direction") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	EvlState& E = *ctx->evl;
	const int nevl = (int)E.dirs.size();
	const size_t per = (size_t)E.nslot * 256;
	if ((r = dev_alloc(ctx, E.opd, per * nevl)) || (r = dev_alloc(ctx, E.sums, (size_t)4 * nevl)) ||
		(r = dev_alloc(ctx, E.coeff, (size_t)3 * nevl)))
		return r;
	if (E.sums_h_n < (size_t)4 * nevl) {
		if (E.sums_h) cudaFreeHost(E.sums_h);
		E.sums_h = nullptr;
		CK(cudaMallocHost(&E.sums_h, sizeof(double) * 4 * nevl));
		E.sums_h_n = (size_t)4 * nevl;
	}
	// (a) ray trace of every direction's tiles (atm2loc, cuda/sim/perfevl.cu:362-364)
	for (int e0 = 0; e0 < nevl; e0 += SHWFS_MAX_ENTRIES) {
		GeomParams gp;
		geom_init(ctx, gp);
		for (int e = e0; e < nevl && e < e0 + SHWFS_MAX_ENTRIES; e++) {
			const auto& d = E.dirs[e];
			if ((r = add_geom_entry(ctx, gp, d.thetax, d.thetay, d.hs, 0, 0, 0, 0, 0, isim, E.torigx.p, E.torigy.p,
					 E.nslot, 16, E.dx, E.opd.p + per * e)))
				return r;
		}
		// the directions of a tile together: the screens' rows are fetched once for all
		gp.interleave = ctx->trace_order != SHWFS_TRACE_LISTED;
		if ((r = launch_geom(ctx, gp))) return r;
	}
	// (b) WFE sums (calc_ptt, cuda/sim/perfevl.cu:46-102)
	CK(cudaMemsetAsync(E.sums.p, 0, sizeof(double) * 4 * nevl, ctx->stream));
	{
		StageMark m(ctx, SHWFS_STAGE_POST);
		const unsigned nblk = (unsigned)((E.nslot + EVL_SUM_TILES - 1) / EVL_SUM_TILES);
		evl_sums_kernel<<<dim3(nblk, nevl), 256, 0, ctx->stream>>>(evl_raster(E), E.opd.p, E.sums.p);
		CK(cudaGetLastError());
	}
	// (c) PSF sums (psfcomp_r, cuda/sim/perfevl.cu:255-300)
	if (do_psf && !E.psf.empty()) {
		if (E.pttr) {
			evl_coeff_kernel<<<(nevl + 127) / 128, 128, 0, ctx->stream>>>(E.sums.p, E.imcc_d.p, E.coeff.p, nevl);
			CK(cudaGetLastError());
		}
		size_t tn = 0;
		for (auto& P : E.psf) tn = std::max(tn, (size_t)nevl * P.psfsize * E.nY);
		if ((r = dev_alloc(ctx, E.T, tn))) return r;
		for (auto& P : E.psf) {
			const size_t pn = (size_t)nevl * P.psfsize * P.psfsize;
			if (P.psf.n != pn) {
				if ((r = dev_alloc(ctx, P.psf, pn))) return r;
				CK(cudaMemsetAsync(P.psf.p, 0, sizeof(float) * pn, ctx->stream));
				E.nframe = 0;
			}
			StageMark m(ctx, SHWFS_STAGE_INTS);
			switch (P.N) {
			case 64: r = evl_launch_psf<64>(ctx, E, P, nevl); break;
			case 128: r = evl_launch_psf<128>(ctx, E, P, nevl); break;
			case 256: r = evl_launch_psf<256>(ctx, E, P, nevl); break;
			case 512: r = evl_launch_psf<512>(ctx, E, P, nevl); break;
			case 1024: r = evl_launch_psf<1024>(ctx, E, P, nevl); break;
			case 2048: r = evl_launch_psf<2048>(ctx, E, P, nevl); break;
			case 4096: r = evl_launch_psf<4096>(ctx, E, P, nevl); break;
			default: r = fail(ctx, SHWFS_EINVAL, "evl: nembed %d", P.N);
			}
			if (r) return r;
		}
		E.nframe++;
	}
	CK(cudaMemcpyAsync(E.sums_h, E.sums.p, sizeof(double) * 4 * nevl, cudaMemcpyDeviceToHost, ctx->stream));
	ctx->d2h_bytes += sizeof(double) * 4 * nevl;
	E.queued = 1;
	return 0;
}

int shwfs_evl_sync(shwfs_ctx* ctx, double* wfe, double* coeff) {
	if (!ctx || !ctx->evl || !ctx->evl->queued)
		return ctx ? fail(ctx, SHWFS_ESTATE, "evl_sync: nothing queued") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	CK(cudaStreamSynchronize(ctx->stream));
	if ((r = check_errflag(ctx))) return r;
	const EvlState& E = *ctx->evl;
	// calc_ptt_post (cuda/sim/perfevl.cu:105-127) / loc_calc_ptt_stride (math/loc.c:692-703)
	for (size_t e = 0; e < E.dirs.size(); e++) {
		const double* s = E.sums_h + 4 * e;
		const double tot = s[0], c[3] = {s[1], s[2], s[3]};
		double cf[3];
		for (int i = 0; i < 3; i++) cf[i] = E.imcc[i] * c[0] + E.imcc[3 + i] * c[1] + E.imcc[6 + i] * c[2];
		const double pis = E.ipcc * c[0] * c[0];
		const double ptt = c[0] * cf[0] + c[1] * cf[1] + c[2] * cf[2];
		if (wfe) {
			wfe[3 * e] = tot - pis;
			wfe[3 * e + 1] = ptt - pis;
			wfe[3 * e + 2] = tot - ptt;
		}
		if (coeff)
			for (int i = 0; i < 3; i++) coeff[3 * e + i] = cf[i];
	}
	return 0;
}

int shwfs_evl_psf_get(shwfs_ctx* ctx, int ievl, int iwvl, double* psf, long* nframe) {
	if (!ctx || !ctx->evl || ievl < 0 || ievl >= (int)ctx->evl->dirs.size() || iwvl < 0 ||
		iwvl >= (int)ctx->evl->psf.size() || !psf)
		return ctx ? fail(ctx, SHWFS_EINVAL, "evl_psf_get: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const EvlPsf& P = ctx->evl->psf[iwvl];
	const int n = P.psfsize;
	std::vector<float> h((size_t)n * n, 0.f);
	if (P.psf.p) {
		CK(cudaMemcpyAsync(h.data(), P.psf.p + (size_t)ievl * n * n, sizeof(float) * n * n, cudaMemcpyDeviceToHost,
			ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
	}
	for (int ax = 0; ax < n; ax++)
		for (int ay = 0; ay < n; ay++) psf[ax + (size_t)ay * n] = h[(size_t)ax * n + ay];
	if (nframe) *nframe = ctx->evl->nframe;
	return 0;
}

int shwfs_evl_opd_dev(shwfs_ctx* ctx, int ievl, float* opd) {
	if (!ctx || !ctx->evl || !opd || ievl < 0 || ievl >= (int)ctx->evl->dirs.size() || !ctx->evl->opd.p)
		return ctx ? fail(ctx, SHWFS_EINVAL, "evl_opd_dev: bad arguments or nothing queued") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const EvlState& E = *ctx->evl;
	evl_gather_kernel<<<(unsigned)((E.nloc + 255) / 256), 256, 0, ctx->stream>>>(
		E.opd.p + (size_t)ievl * E.nslot * 256, E.loc_addr.p, E.nloc, opd);
	CK(cudaGetLastError());
	return 0;
}

}  // extern "C"
