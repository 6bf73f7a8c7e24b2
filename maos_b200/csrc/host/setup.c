/*
 * Setup producers of the Shack-Hartmann frame (declared in
 * include/shwfs_setup.h).  Each step restates the reference routine cited at
 * its head, in double precision, with the reference's operation order where
 * the result is compared bit for bit (geometry, valid mask, pixel map).
 */
#include "../../../include/shwfs_setup.h"
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hmath.h"

#define EPS_REF 1.e-15 /* sys/common.h:62 (double build) */

struct shwfs_setup {
	shwfs_setup_cfg cfg;
	char err[256];
	int nsa, nopd, notf, pixpsax, pixpsay, npix, llt_nx;
	double dx, areascale, dtheta, i0sumsum;
	double saasum;     /* powfs.saasum as the reference forms it (see setup_geom) */
	double *salocx, *salocy, *origx, *origy, *amp, *saa;
	double* nominal;   /* notf^2 */
	int* simap_idx;    /* npix*4 */
	double* simap_wt;  /* npix*4 */
	double *srot, *srsa;
	hcplx* etf;        /* nsa*notf^2 */
	double* lltamp;    /* llt_nx^2 */
	double llt_orig;
	double *mtche, *i0sum, *i0, *gx, *gy;
	double* sepsf;     /* nsa*notf^2 short-exposure PSF (matched filter only) */
	hcplx* seotf;      /* nsa*notf^2 its OTF / notf^2, peak in the corner */
};

static int serr(shwfs_setup* s, const char* fmt, ...) {
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(s->err, sizeof(s->err), fmt, ap);
	va_end(ap);
	return SHWFS_EINVAL;
}

/* math/mathdef.h sinc, evaluated as the macro expands. */
static double sinc_ref(double a, double b) {
	const double x = a * b;
	return x != 0 ? (sin(M_PI * a * b) / (M_PI * a * b)) : 1;
}

/* math/loc.c:942-986 loc_circle_add for one point of sampling dx. */
static double circle_add_pt(double x, double y, double dx, double r, double val) {
	const int nres = 10;
	const double cres = (nres - 1.) / 2.;
	const double res = 1. / nres;
	const double dxres = res * dx, res2 = res * res;
	const double r2 = r * r;
	const double r2l = (r - dx * 1.5) * (r - dx * 1.5);
	const double r2u = (r + dx * 1.5) * (r + dx * 1.5);
	const double r2r = pow(x, 2) + pow(y, 2);
	if (r2r < r2l) return val;
	if (r2r < r2u) {
		long tot = 0;
		for (int jres = 0; jres < nres; jres++) {
			const double iiy = y + (jres - cres) * dxres;
			const double rr2y = iiy * iiy;
			for (int ires = 0; ires < nres; ires++) {
				const double iix = x + (ires - cres) * dxres;
				if (iix * iix + rr2y <= r2) tot++;
			}
		}
		return (double)tot * res2 * val;
	}
	return 0;
}

/* math/mathmisc.c:109 nextfftsize: smallest even n' >= n with only 2,3,5,7 factors. */
static long nextfftsize(long n) {
	if (n == 0) n = 1;
	n = (n + 1) / 2 * 2;
	for (;; n += 2) {
		long m = n;
		const int rad[4] = {2, 3, 5, 7};
		for (int i = 0; i < 4; i++)
			while (m % rad[i] == 0) m /= rad[i];
		if (m == 1) return n;
	}
}

/* ---- geometry: maos/powfs.c:256-462 (setup_shwfs_geom), :141-237 (sa_reduce) ---- */
static int setup_geom(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	const int order = c->order;
	const double dsa = c->dsa;
	const double areafulli = order > 2 ? 1. : 4. / M_PI;
	const int nxsa = 2 * (int)round(0.5 * dsa / c->dx);
	const double dx = dsa / nxsa;
	const double dxoffset = dx * 0.5;
	const double offset = (order & 1) ? -0.5 : 0;
	const int orderpad = (int)(order + (order > 2 ? (1 + 0. / dsa) * 2 : 0));
	const double r2max = pow(order * 0.5, 2);
	const double r2min = dsa < c->Din ? pow(c->Din / dsa / 2, 2) : -1;
	const int jmin = -orderpad / 2, jmax = (orderpad - 1) / 2;
	const int nside = jmax - jmin + 1;
	const long ntot = (long)nside * nside;
	const int npsa = nxsa * nxsa;
	double* sx = malloc(sizeof(double) * ntot);
	double* sy = malloc(sizeof(double) * ntot);
	int* gi = malloc(sizeof(int) * ntot); /* grid column of each candidate */
	int* gj = malloc(sizeof(int) * ntot);
	long count = 0;
	for (int j = jmin; j <= jmax; j++) {
		for (int i = jmin; i <= jmax; i++) {
			const double xc = (double)i + offset, yc = (double)j + offset;
			const double r1 = pow(xc + 1, 2) + pow(yc + 1, 2);
			const double r2 = pow(xc + 1, 2) + pow(yc, 2);
			const double r3 = pow(xc, 2) + pow(yc + 1, 2);
			const double r4 = pow(xc, 2) + pow(yc, 2);
			if (r1 < r2max || r2 < r2max || r3 < r2max || r4 < r2max || r1 > r2min || r2 > r2min || r3 > r2min ||
				r4 > r2min) {
				sx[count] = xc * dsa;
				sy[count] = yc * dsa;
				gi[count] = i - jmin;
				gj[count] = j - jmin;
				count++;
			}
		}
	}
	/* amplitude on every OPD point (mkamp, maos/utils.c:497-508) and area */
	double* amp = calloc((size_t)count * npsa, sizeof(double));
	double* saa = calloc(count, sizeof(double));
	for (long isa = 0; isa < count; isa++) {
		const double ox = sx[isa] + dxoffset, oy = sy[isa] + dxoffset;
		double area = 0;
		for (int jj = 0; jj < nxsa; jj++) {
			const double yy = oy + (double)jj * dx;
			for (int ii = 0; ii < nxsa; ii++) {
				const double xx = ox + (double)ii * dx;
				double a;
				if (c->amp_binary) {
					const double r2 = pow(xx, 2) + pow(yy, 2);
					a = (r2 <= 0.25 * c->D * c->D && r2 >= 0.25 * c->Din * c->Din) ? 1 : 0;
				} else {
					a = circle_add_pt(xx, yy, dx, c->D * 0.5, 1);
					if (c->Din > 0) a += circle_add_pt(xx, yy, dx, c->Din * 0.5, -1);
				}
				amp[isa * npsa + jj * nxsa + ii] = a;
				area += a * a;
			}
		}
		saa[isa] = area * (1. / (double)npsa);
		if (fabs(areafulli - 1) > EPS_REF) saa[isa] *= areafulli;
	}
	/* sa_reduce: drop subapertures with two or fewer valid neighbours, then
	   those under the area threshold.  The candidate grid is full, so grid
	   coordinates give the neighbour map directly. */
	const double saat = c->saat;
	if (saat > 0 && count > 4) {
		int* map = malloc(sizeof(int) * ntot);
		for (long k = 0; k < ntot; k++) map[k] = -1;
		for (long isa = 0; isa < count; isa++) map[gi[isa] + gj[isa] * nside] = (int)isa;
		int changed;
		do {
			changed = 0;
			for (long isa = 0; isa < count; isa++) {
				int nedge = 0, ncorner = 0;
				const int nself = saa[isa] >= saat;
				for (int jx = -1; jx < 2; jx++) {
					for (int jy = -1; jy < 2; jy++) {
						if (jx == 0 && jy == 0) continue;
						const int ix = gi[isa] + jx, iy = gj[isa] + jy;
						if (ix < 0 || iy < 0 || ix >= nside || iy >= nside) continue;
						const int jsa = map[ix + iy * nside];
						if (jsa >= 0 && saa[jsa] >= saat) {
							if (abs(jx + jy) == 1) nedge++;
							else ncorner++;
						}
					}
				}
				if (nself && ncorner + nedge <= 2) {
					saa[isa] = 0;
					changed++;
				}
			}
		} while (changed);
		free(map);
	}
	long nsa = 0;
	for (long isa = 0; isa < count; isa++) {
		if (saat > 0 && !(saa[isa] >= saat)) continue;
		if (nsa != isa) {
			sx[nsa] = sx[isa];
			sy[nsa] = sy[isa];
			saa[nsa] = saa[isa];
			memmove(amp + nsa * npsa, amp + isa * npsa, sizeof(double) * npsa);
		}
		nsa++;
	}
	free(gi);
	free(gj);
	/* powfs.saasum (maos/powfs.c:227-230) is summed before saa is cut to the
	   kept subapertures: over all candidates after the compaction, the
	   entries past the kept ones included */
	s->saasum = 0;
	for (long isa = 0; isa < count; isa++) s->saasum += saa[isa];
	if (nsa == 0) {
		free(sx); free(sy); free(amp); free(saa);
		return serr(s, "no subaperture above the area threshold");
	}
	s->nsa = (int)nsa;
	s->nopd = nxsa;
	s->dx = dx;
	s->areascale = areafulli;
	s->salocx = realloc(sx, sizeof(double) * nsa);
	s->salocy = realloc(sy, sizeof(double) * nsa);
	s->origx = malloc(sizeof(double) * nsa);
	s->origy = malloc(sizeof(double) * nsa);
	for (long i = 0; i < nsa; i++) {
		s->origx[i] = s->salocx[i] + dxoffset;
		s->origy[i] = s->salocy[i] + dxoffset;
	}
	s->amp = realloc(amp, sizeof(double) * nsa * npsa);
	s->saa = realloc(saa, sizeof(double) * nsa);
	return 0;
}

/* ---- maos/powfs.c:725-885 (setup_shwfs_prep_phy) ---- */
static int setup_prep_phy(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	s->pixpsax = s->pixpsay = c->pixpsa;
	s->npix = s->pixpsax * s->pixpsay;
	const double safov = fmax(s->pixpsax * c->pixtheta, s->pixpsay * c->pixtheta);
	const double dtheta = c->wvl / (c->dsa * c->embfac);
	if (c->notf) {
		s->notf = (c->notf + 1) / 2 * 2;
	} else {
		long n = (long)fmax(s->nopd * c->embfac, ceil(safov / dtheta));
		s->notf = (int)nextfftsize(n);
	}
	if (c->has_llt) {
		s->srot = malloc(sizeof(double) * s->nsa);
		s->srsa = malloc(sizeof(double) * s->nsa);
		const double ox2 = c->llt_ox - c->dsa * 0.5;
		const double oy2 = c->llt_oy - c->dsa * 0.5;
		for (int isa = 0; isa < s->nsa; isa++) {
			const double ddx = s->salocx[isa] - ox2, ddy = s->salocy[isa] - oy2;
			s->srot[isa] = atan2(ddy, ddx);
			s->srsa[isa] = sqrt(pow(ddx, 2) + pow(ddy, 2));
		}
	}
	return 0;
}

/* ---- DTF nominal and pixel map: lib/mkdtf.c:26-80 (cotf_treat, dtf_otf),
        :89-184 (mkdtf), lib/mkh.c:62-150 (mkht) ---- */
static int setup_dtf(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	const int n = s->notf, n2 = n >> 1;
	const double dtheta = c->wvl / (c->dsa * c->embfac);
	s->dtheta = dtheta;
	const double pdx = c->pixtheta / dtheta, pdy = c->pixtheta / dtheta;
	const double duxp = pdx / n, duyp = pdy / n;
	const double pixblur = fabs(c->pixblur);
	const double bxp2 = -2 * pow(M_PI * pixblur * duxp, 2);
	const double byp2 = -2 * pow(M_PI * pixblur * duyp, 2);
	hcplx* w = malloc(sizeof(hcplx) * n * n);
	for (int iy = 0; iy < n; iy++) {
		const long jy = iy - n2;
		for (int ix = 0; ix < n; ix++) {
			const long jx = ix - n2;
			const double ir = 1. * jx + 0. * jy;
			const double ia = -0. * jx + 1. * jy;
			const double v = (pdx ? sinc_ref(ir, duxp) * sinc_ref(ia, duyp) * pdx * pdy : 1) *
				(pixblur ? exp(bxp2 * (ir * ir) + byp2 * (ia * ia)) : 1);
			w[ix + iy * n] = v;
		}
	}
	/* treat: fftshift, FFT(-1), fftshift, FFT(+1), /n^2, real part */
	hfftshift(w, n, n);
	hfft2(w, n, n, -1);
	hfftshift(w, n, n);
	hfft2(w, n, n, 1);
	s->nominal = malloc(sizeof(double) * n * n);
	for (int i = 0; i < n * n; i++) s->nominal[i] = creal(w[i] * (1. / (double)(n * n)));
	free(w);
	/* pixel map: bilinear taps of each pixel centre on the PSF grid */
	const double pxo = -(s->pixpsax * 0.5 - 0.5) * c->pixtheta;
	const double pyo = -(s->pixpsay * 0.5 - 0.5) * c->pixtheta;
	const double psf_ox = -n2 * dtheta; /* loc_psf origin = map origin */
	const double dx_in1 = 1. / dtheta;
	const double dispx = (0 - psf_ox) * dx_in1, dispy = (0 - psf_ox) * dx_in1;
	s->simap_idx = malloc(sizeof(int) * s->npix * 4);
	s->simap_wt = malloc(sizeof(double) * s->npix * 4);
	const double ct = cos(-0.), st = sin(-0.);
	for (int iy = 0; iy < s->pixpsay; iy++) {
		const double py = iy * c->pixtheta + pyo;
		for (int ix = 0; ix < s->pixpsax; ix++) {
			const double px = ix * c->pixtheta + pxo;
			const int p = ix + iy * s->pixpsax;
			const double x2 = ct * px + st * py;
			const double y2 = -st * px + ct * py;
			double fx1 = x2 * dx_in1 + dispx, fy1 = y2 * dx_in1 + dispy;
			const int nplocx = (int)floor(fx1), nplocy = (int)floor(fy1);
			fx1 -= nplocx;
			fy1 -= nplocy;
			const double fx[2] = {1. - fx1, fx1}, fy[2] = {1. - fy1, fy1};
			int k = 0;
			for (int jy = 0; jy < 2; jy++) {
				for (int jx = 0; jx < 2; jx++) {
					const double weight = fx[jx] * fy[jy];
					const int gx = nplocx + jx, gy = nplocy + jy;
					if (weight > EPS_REF && gx >= 0 && gx < n && gy >= 0 && gy < n) {
						s->simap_idx[4 * p + k] = gx + gy * n;
						s->simap_wt[4 * p + k] = weight;
						k++;
					}
				}
			}
			for (; k < 4; k++) {
				s->simap_idx[4 * p + k] = -1;
				s->simap_wt[4 * p + k] = 0;
			}
		}
	}
	return 0;
}

/* ---- ETF: lib/mkdtf.c:186-396 (mketf, interpolation path, one LLT) ---- */
static int setup_etf(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	const int nhp = c->na_n;
	if (nhp < 2 || !c->na_h || !c->na_p) return serr(s, "LGS needs a sodium profile of at least 2 samples");
	const double* px = c->na_h;
	const double* pna = c->na_p;
	const double cosza = 1, htel = 0;
	const double hpmin = (px[0] - htel) / cosza;
	const double dhp1 = cosza / (px[1] - px[0]);
	if (fabs((px[nhp - 1] - px[0]) / ((nhp - 1) * (px[1] - px[0])) - 1.) > 1.e-3)
		return serr(s, "the sodium profile is not evenly spaced");
	double i0scale = 0;
	for (int i = 0; i < nhp; i++) i0scale += pna[i];
	const int n = s->notf, n2 = n >> 1;
	const double dtheta = s->dtheta;
	const int npad = 2, nover = 2;
	const int netf = n * nover * npad;
	const double dtetf = dtheta / nover;
	const double dusc = (netf * dtetf) / (dtheta * n);
	const int netf2 = netf >> 1;
	const int etf0 = netf2 - (int)round(n2 * (dtheta / dtetf));
	const int etf1 = etf0 + (int)round(n * (dtheta / dtetf));
	if (etf0 < 0) return serr(s, "invalid ETF configuration");
	double* thetas = calloc(netf, sizeof(double));
	for (int it = etf0; it < etf1; it++) thetas[it] = (it - netf2) * dtetf;
	const double hs = c->hs;
	s->etf = calloc((size_t)s->nsa * n * n, sizeof(hcplx));
	hcplx* etf = malloc(sizeof(hcplx) * netf);
	for (int isa = 0; isa < s->nsa; isa++) {
		hcplx* e2 = s->etf + (size_t)isa * n * n;
		const double rsa = s->srsa[isa];
		double etf2sum = 0;
		if (!rsa) {
			for (int i = 0; i < n * n; i++) e2[i] = 1;
		} else {
			for (int i = 0; i < netf; i++) etf[i] = 0;
			for (int icomp = etf0; icomp < etf1; icomp++) {
				const double itheta = thetas[icomp];
				const double ih = hs * rsa / (rsa + itheta * hs);
				const double iih = (ih - hpmin) * dhp1;
				const int iihf = (int)floor(iih);
				const double iihw = iih - iihf;
				if (iihf < 0 || iihf > nhp - 2) {
					etf[icomp] = 0.;
				} else {
					const double tmp = pna[iihf] * (1. - iihw) + pna[iihf + 1] * iihw;
					etf[icomp] = tmp;
					etf2sum += tmp;
				}
			}
		}
		if (etf2sum) {
			for (int i = 0; i < netf; i++) etf[i] *= i0scale / etf2sum;
			hfftshift(etf, netf, 1);
			hfft2(etf, netf, 1, -1);
			hfftshift(etf, netf, 1);
			const double theta = s->srot[isa];
			const double ct = cos(theta), st = sin(theta);
			for (int icompy = 0; icompy < n; icompy++) {
				const double iy = (icompy - n2);
				for (int icompx = 0; icompx < n; icompx++) {
					const double ix = (icompx - n2);
					double ir = (dusc * (ct * ix + st * iy)) + netf2;
					const int iir = (int)floor(ir);
					ir = ir - iir;
					if (iir >= 0 && iir < netf - 1) {
						e2[icompx + icompy * n] = etf[iir] * (1. - ir) + etf[iir + 1] * ir;
					}
				}
			}
			hfftshift(e2, n, n);
		}
		/* fuse the nominal (lib/mkdtf.c:388-393) */
		for (int i = 0; i < n * n; i++) e2[i] *= s->nominal[i];
	}
	free(etf);
	free(thetas);
	return 0;
}

/* ---- LLT pupil amplitude: maos/powfs.c:1183-1232 (setup_powfs_llt) ---- */
static int setup_llt(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	const double lltd = c->llt_d;
	const double dx = s->dx;
	double lltdsa = fmax(lltd, c->dsa);
	const int nxsa = (int)round(lltdsa / dx);
	lltdsa = dx * nxsa;
	const double o = (dx - lltdsa) * 0.5;
	s->llt_nx = nxsa;
	s->llt_orig = o;
	s->lltamp = calloc((size_t)nxsa * nxsa, sizeof(double));
	const double l2max = pow(lltd * 0.5, 2);
	const double r2waist = pow(lltd * 0.5 * c->llt_widthp, 2);
	double sumamp2 = 0;
	for (int iy = 0; iy < nxsa; iy++) {
		const double yy = iy * dx + o;
		for (int ix = 0; ix < nxsa; ix++) {
			const double xx = ix * dx + o;
			const double r2 = xx * xx + yy * yy;
			const double r2m = pow(xx - 0, 2) + pow(yy - 0, 2);
			const double a = exp(-r2m / r2waist);
			sumamp2 += pow(a, 2);
			if (r2 <= l2max) s->lltamp[iy * nxsa + ix] = a;
		}
	}
	sumamp2 = 1. / (sqrt(sumamp2));
	for (int i = 0; i < nxsa * nxsa; i++) s->lltamp[i] *= sumamp2;
	return 0;
}

/* ---- short-exposure OTF of the turbulence (lib/genotf.c, lib/gensei.c:41-209) ---- */

/* Modified Bessel function of the second kind K_nu(x), x > 0, from its
   integral representation K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt
   (DLMF 10.32.9) by the trapezoidal rule: the integrand is analytic in the
   strip |Im t| < pi/2 and decays double-exponentially, so the rule converges
   exponentially (error ~ exp(-pi^2 / h)); h = 1/32 is far below double
   precision. */
static double bessel_k(double nu, double x) {
	const double h = 1. / 32;
	double s = 0.5 * exp(-x);
	for (int k = 1; k < 1000000; k++) {
		const double t = k * h;
		const double term = exp(-x * cosh(t)) * cosh(nu * t);
		s += term;
		if (term < 1e-20 * s) break;
	}
	return s * h;
}

/* Phase covariance (m^2 of OPD, r0 at 0.5 um) at separation r, as turbcov
   (lib/turbulence.c:400-435) defines it with rmax = 0: von Karman for finite
   L0, Kolmogorov structure function otherwise. */
static double turb_cov(double r, double r0, double L0) {
	const double k05 = pow(2 * M_PI / 0.5e-6, -2);
	if (!isfinite(L0)) return -0.5 * 6.88 * k05 * pow(r0, -5. / 3.) * pow(r, 5. / 3.);
	const double tg1 = tgamma(11. / 6) * pow(24. / 5 * tgamma(6. / 5.), 5. / 6.) * k05 / pow(M_PI, 8. / 3.);
	const double f0 = 1. / L0, r0f0p = pow(r0 * f0, -5. / 3.);
	if (fabs(r) < EPS_REF) return tg1 * tgamma(5. / 6.) / 2 * r0f0p;
	const double x = r * 2 * M_PI * f0;
	return tg1 / pow(2, 5. / 6.) * r0f0p * pow(x, 5. / 6.) * bessel_k(5. / 6., x);
}

/* Inverse of a symmetric matrix by its eigen-decomposition with the
   thresholds of svd_pow(A, -1) (math/blas.c:441-481: 1e-7 absolute, 1e-3
   relative to the previous kept value). a is destroyed. */
static void pinv_sym(double* a, int n, double* out) {
	double w[16], v[256];
	int order[16];
	hsyev_jacobi(a, n, w, v);
	for (int i = 0; i < n; i++) order[i] = i;
	for (int i = 0; i < n; i++)
		for (int j = i + 1; j < n; j++)
			if (fabs(w[order[j]]) > fabs(w[order[i]])) {
				const int t = order[i];
				order[i] = order[j];
				order[j] = t;
			}
	const double maxeig = fabs(w[order[0]]);
	double thres2 = 1e-3 * maxeig, sinv[16] = {0};
	for (int k = 0; k < n; k++) {
		const double sv = fabs(w[order[k]]);
		if (sv > 1e-7 * maxeig && sv > thres2) {
			thres2 = sv * 1e-3;
			sinv[k] = 1. / w[order[k]];
		} else {
			break;
		}
	}
	for (int i = 0; i < n; i++)
		for (int j = 0; j < n; j++) {
			double s = 0;
			for (int k = 0; k < n; k++) s += v[i + order[k] * n] * sinv[k] * v[j + order[k] * n];
			out[i + j * n] = s;
		}
}

/* The tip/tilt-removed short-exposure OTF of one pupil of nx x nx points
   (spacing dx, amplitude a) for a Kolmogorov/von Karman covariance B of the
   pupil points (nloc x nloc): genotf_do (lib/genotf.c:46-108) with pttr.
   Piston, tip and tilt are removed from both sides of B with the amplitude
   weighting (loc_remove_ptt with cov, math/loc.c:794-826), then
   OTF(m) = sum over point pairs (i, i+m) of a_i a_{i+m} e^{k^2 B'_{i,i+m}}
   / sqrt(e^{k^2 B'_ii} e^{k^2 B'_jj}) / sum a^2, on npsf x npsf separations
   with the zero separation at (npsf/2, npsf/2).  out: npsf^2, x fastest. */
static void genotf_pupil(const double* B, int nx, double dx, const double* a, double wvl, int npsf, double* out) {
	const int nloc = nx * nx;
	double* BP = malloc(sizeof(double) * nloc * nloc);
	memcpy(BP, B, sizeof(double) * nloc * nloc);
	double* X = malloc(sizeof(double) * nloc);
	double* Y = malloc(sizeof(double) * nloc);
	for (int iy = 0; iy < nx; iy++)
		for (int ix = 0; ix < nx; ix++) {  /* mksqloc_auto (math/loc.c:526-528) */
			X[ix + iy * nx] = ix * dx - nx / 2 * dx;
			Y[ix + iy * nx] = iy * dx - nx / 2 * dx;
		}
	double mcc[9] = {0}, imcc[9];
	for (int i = 0; i < nloc; i++) {
		const double m[3] = {1, X[i], Y[i]};
		for (int r = 0; r < 3; r++)
			for (int c = 0; c < 3; c++) mcc[r + 3 * c] += m[r] * m[c] * a[i];
	}
	pinv_sym(mcc, 3, imcc);
	for (int pass = 0; pass < 2; pass++) {  /* columns, then rows */
		for (int ic = 0; ic < nloc; ic++) {
			const long s0 = pass ? ic : (long)ic * nloc, st = pass ? nloc : 1;
			double c[3] = {0, 0, 0};
			for (int i = 0; i < nloc; i++) {
				const double v = BP[s0 + i * st] * a[i];
				c[0] += v;
				c[1] += v * X[i];
				c[2] += v * Y[i];
			}
			double t[3];
			for (int r = 0; r < 3; r++) t[r] = imcc[r] * c[0] + imcc[r + 3] * c[1] + imcc[r + 6] * c[2];
			for (int i = 0; i < nloc; i++) BP[s0 + i * st] -= t[0] + t[1] * X[i] + t[2] * Y[i];
		}
	}
	const double k2 = pow(2 * M_PI / wvl, 2);
	double* D = malloc(sizeof(double) * nloc);
	for (long k = 0; k < (long)nloc * nloc; k++) BP[k] = exp(k2 * BP[k]);
	for (int i = 0; i < nloc; i++) D[i] = pow(BP[i + (long)i * nloc], -0.5);
	double an = 0;
	for (int i = 0; i < nloc; i++) an += a[i] * a[i];
	an = 1. / an;
	const int h = npsf / 2;
	for (int jm = 0; jm < npsf; jm++)
		for (int im = 0; im < npsf; im++) {
			const int sx = im - h, sy = jm - h;
			double acc = 0;
			for (int iy = 0; iy < nx; iy++) {
				const int jy = iy + sy;
				if (jy < 0 || jy >= nx) continue;
				for (int ix = 0; ix < nx; ix++) {
					const int jx = ix + sx;
					if (jx < 0 || jx >= nx) continue;
					const int i1 = ix + iy * nx, i2 = jx + jy * nx;
					acc += D[i1] * D[i2] * BP[i2 + (long)i1 * nloc] * a[i1] * a[i2];
				}
			}
			out[im + jm * npsf] = acc * an;
		}
	free(BP); free(X); free(Y); free(D);
}

/* Short-exposure PSF and OTF of every subaperture for the matched filter:
   genseotf (lib/gensei.c:41-111: a subaperture of area saa > 1 - 1e-10 takes
   the OTF of the first fullest one, one of area <= 0.01 none), the LLT's OTF
   (genseotf of the LLT pupil), gensepsf (lib/gensei.c:135-209: OTF times the
   conjugate uplink OTF, to the PSF, real part times saa / n^2) and the first
   steps of gensei (:327-335: back to the OTF, times 1/n^2). */
static int setup_seotf(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	const int nopd = s->nopd, n = s->notf, nsa = s->nsa, nloc = nopd * nopd;
	const int npsf = nopd * c->embfac;
	if (npsf != n) return serr(s, "matched-filter setup needs notf == nopd*embfac");
	if (nloc > 4096) return serr(s, "matched-filter setup: at most 64x64 OPD points per subaperture");
	const int turb = c->r0 > 0 && isfinite(c->r0);
	/* the covariance of the pupil points (loc_sep + turbcov, lib/genotf.c:216-227) */
	double* B = calloc((size_t)nloc * nloc, sizeof(double));
	if (turb) {
		double* cov = malloc(sizeof(double) * nopd * nopd);  /* by |dx|, |dy| in points */
		for (int dy = 0; dy < nopd; dy++)
			for (int dx = 0; dx < nopd; dx++)
				cov[dx + dy * nopd] = turb_cov(sqrt(pow(dx * s->dx, 2) + pow(dy * s->dx, 2)), c->r0, c->L0);
		for (int j = 0; j < nloc; j++)
			for (int i = 0; i < nloc; i++)
				B[i + (long)j * nloc] = cov[abs(i % nopd - j % nopd) + abs(i / nopd - j / nopd) * nopd];
		free(cov);
	}
	double* otf = calloc((size_t)nsa * n * n, sizeof(double));
	int isafull = -1;
	double maxarea = 0;
	for (int isa = 0; isa < nsa; isa++)
		if (s->saa[isa] > maxarea) {
			maxarea = s->saa[isa];
			isafull = isa;
		}
	double* full = NULL;
	if (isafull > 0) {  /* as lib/genotf.c:248: the first subaperture cannot be the template */
		full = malloc(sizeof(double) * n * n);
		genotf_pupil(B, nopd, s->dx, s->amp + (size_t)isafull * nloc, c->wvl, n, full);
	}
	const double thres = 1 - 1e-10;
	for (int isa = 0; isa < nsa; isa++) {
		double* o = otf + (size_t)isa * n * n;
		if (full && s->saa[isa] > thres) memcpy(o, full, sizeof(double) * n * n);
		else if (s->saa[isa] > 0.01) genotf_pupil(B, nopd, s->dx, s->amp + (size_t)isa * nloc, c->wvl, n, o);
	}
	free(full);
	free(B);
	double* lotf = NULL;
	if (c->has_llt) {
		const int nl = s->llt_nx, nll = nl * nl;
		if (nl * c->embfac != n) {
			free(otf);
			return serr(s, "LLT pupil size incompatible with notf");
		}
		double* BL = calloc((size_t)nll * nll, sizeof(double));
		if (turb)
			for (int j = 0; j < nll; j++)
				for (int i = 0; i < nll; i++) {
					const double ddx = (i % nl - j % nl) * s->dx, ddy = (i / nl - j / nl) * s->dx;
					BL[i + (long)j * nll] = turb_cov(sqrt(ddx * ddx + ddy * ddy), c->r0, c->L0);
				}
		lotf = malloc(sizeof(double) * n * n);
		genotf_pupil(BL, nl, s->dx, s->lltamp, c->wvl, n, lotf);
		free(BL);
	}
	s->sepsf = calloc((size_t)nsa * n * n, sizeof(double));
	s->seotf = malloc(sizeof(hcplx) * nsa * n * n);
	hcplx* t = malloc(sizeof(hcplx) * n * n);
	const double n2 = (double)n * n;
	for (int isa = 0; isa < nsa; isa++) {
		const double* o = otf + (size_t)isa * n * n;
		/* the OTFs are real (no static aberration): o * conj(lotf) */
		for (int i = 0; i < n * n; i++) t[i] = o[i] * (lotf ? lotf[i] : 1.);
		hfftshift(t, n, n);
		hfft2(t, n, n, 1);
		hfftshift(t, n, n);
		double* ps = s->sepsf + (size_t)isa * n * n;
		const double norm = s->saa[isa] / n2;
		for (int i = 0; i < n * n; i++) ps[i] = creal(t[i]) * norm;
		hcplx* so = s->seotf + (size_t)isa * n * n;
		for (int i = 0; i < n * n; i++) so[i] = ps[i];
		hfftshift(so, n, n);
		hfft2(so, n, n, -1);
		for (int i = 0; i < n * n; i++) so[i] *= 1. / n2;
	}
	free(t);
	free(otf);
	free(lotf);
	return 0;
}

/* |FFT(embed(amp))|^2 scaled, then FFT: the OTF of a flat wavefront
   (maos/wfsints.c:233-260 with zero OPD). a: nopd^2; out: n^2, peak in corner. */
static void flat_otf(const double* a, int nopd, int n, double scale, hcplx* out) {
	const int pad = (n - nopd) / 2;
	for (int i = 0; i < n * n; i++) out[i] = 0;
	for (int iy = 0; iy < nopd; iy++)
		for (int ix = 0; ix < nopd; ix++) out[(iy + pad) * n + ix + pad] = a[iy * nopd + ix];
	hfft2(out, n, n, -1);
	for (int i = 0; i < n * n; i++) out[i] = (creal(out[i]) * creal(out[i]) + cimag(out[i]) * cimag(out[i])) * scale;
	hfft2(out, n, n, -1);
}

/* ---- i0/gx/gy of a flat wavefront (lib/gensei.c:213-419 with the
        diffraction-limited short-exposure OTF) and the matched filter
        (lib/mtch.c:93-211 mtch, :223-335 mtch_cell) ---- */
static int setup_mtch(shwfs_setup* s) {
	const shwfs_setup_cfg* c = &s->cfg;
	const int n = s->notf, n2 = n >> 1, nopd = s->nopd, npix = s->npix, nsa = s->nsa;
	if (nopd * c->embfac != n) return serr(s, "matched-filter setup needs notf == nopd*embfac");
	const double nwvf = (double)nopd * c->embfac;
	const double norm_psf = sqrt(s->areascale) / ((double)nopd * nwvf);
	const double norm_ints = c->siglev * norm_psf * norm_psf / ((double)n * n);
	const double dux = 1. / (s->dtheta * n);
	hcplx* Ux = malloc(sizeof(hcplx) * n);
	for (int ix = 0; ix < n; ix++) {
		const int jx = ix < n2 ? ix : (ix - n);
		Ux[ix] = I * (-2. * M_PI * jx * dux);
	}
	hcplx* lotf = NULL;
	if (c->has_llt) {
		const int nl = s->llt_nx;
		const int nlw = nl * c->embfac;
		if (nlw != n) return serr(s, "LLT pupil size incompatible with notf");
		lotf = malloc(sizeof(hcplx) * n * n);
		flat_otf(s->lltamp, nl, n, 1. / ((double)nlw * nlw), lotf);
	}
	s->i0 = calloc((size_t)nsa * npix, sizeof(double));
	s->gx = calloc((size_t)nsa * npix, sizeof(double));
	s->gy = calloc((size_t)nsa * npix, sizeof(double));
	hcplx* otf = malloc(sizeof(hcplx) * n * n);
	hcplx* t = malloc(sizeof(hcplx) * n * n);
	/* the matched filter starts from the short-exposure OTF (gensei, lib/gensei.c:327-366), scaled
	   by the signal level; the CoG's i0 sums from the diffraction-limited frame */
	const double scale = s->seotf ? c->siglev : norm_ints;
	for (int isa = 0; isa < nsa; isa++) {
		if (s->seotf) {
			memcpy(otf, s->seotf + (size_t)isa * n * n, sizeof(hcplx) * n * n);
		} else {
			flat_otf(s->amp + (size_t)isa * nopd * nopd, nopd, n, 1, otf);
			if (lotf)
				for (int i = 0; i < n * n; i++) otf[i] *= conj(lotf[i]);
		}
		if (s->etf) {
			const hcplx* e = s->etf + (size_t)isa * n * n;
			for (int i = 0; i < n * n; i++) otf[i] *= e[i];
		} else {
			for (int i = 0; i < n * n; i++) otf[i] *= s->nominal[i];
		}
		for (int d = 0; d < 3; d++) {
			double* out = d == 0 ? s->i0 : d == 1 ? s->gx : s->gy;
			for (int iy = 0; iy < n; iy++)
				for (int ix = 0; ix < n; ix++) {
					const hcplx f = d == 0 ? 1 : d == 1 ? Ux[ix] : Ux[iy];
					t[ix + iy * n] = otf[ix + iy * n] * f;
				}
			hfft2(t, n, n, 1);
			out += (size_t)isa * npix;
			for (int p = 0; p < npix; p++) {
				double v = 0;
				for (int k = 0; k < 4; k++) {
					const int id = s->simap_idx[4 * p + k];
					if (id >= 0) v += s->simap_wt[4 * p + k] * creal(t[id]);
				}
				out[p] = v * scale;
			}
		}
	}
	free(otf);
	free(t);
	free(lotf);
	free(Ux);
	/* matched filter */
	s->i0sum = malloc(sizeof(double) * nsa);
	double i0max = 0;
	for (int isa = 0; isa < nsa; isa++) {
		double sum = 0;
		for (int p = 0; p < npix; p++) sum += s->i0[(size_t)isa * npix + p];
		s->i0sum[isa] = sum;
		if (sum > i0max) i0max = sum;
	}
	s->i0sumsum = 0;
	for (int isa = 0; isa < nsa; isa++) s->i0sumsum += s->i0sum[isa];
	if (c->gradtype != SHWFS_GRAD_MF) return 0;
	const double i0thres = fmax(i0max * 0.1, 10 * c->rne);
	const double kpx = 1. / c->pixtheta, kpy = 1. / c->pixtheta;
	const double bkgrnd_res = c->bkgrnd - c->bkgrndc;
	const double rne2 = c->rne * c->rne;
	const double nea2thres = c->pixtheta * c->pixtheta * 100;
	int nmod = 3, crx = 0, cry = 0;
	if (c->mtchcr == 1 || c->mtchcr == 2) {
		crx = nmod;
		nmod += 2;
	}
	if (c->mtchcr == 1 || c->mtchcr == 3) {
		cry = nmod;
		nmod += 2;
	}
	s->mtche = calloc((size_t)nsa * 2 * npix, sizeof(double));
	double* A = malloc(sizeof(double) * npix * nmod);
	double* wt = malloc(sizeof(double) * npix);
	double* cc = malloc(sizeof(double) * nmod * nmod);
	double* ev = malloc(sizeof(double) * nmod * nmod);
	double* ew = malloc(sizeof(double) * nmod);
	double* inv = malloc(sizeof(double) * nmod * nmod);
	double* P = malloc(sizeof(double) * nmod * npix);
	double i0m[2 * 7];
	for (int k = 0; k < 2 * 7; k++) i0m[k] = 0;
	i0m[0 + 2 * 0] = 1;
	i0m[1 + 2 * 1] = 1;
	if (crx) {
		i0m[0 + 2 * crx] = cos(0.);
		i0m[1 + 2 * crx] = sin(0.);
		i0m[0 + 2 * (crx + 1)] = -i0m[0 + 2 * crx];
		i0m[1 + 2 * (crx + 1)] = -i0m[1 + 2 * crx];
	}
	if (cry) {
		i0m[0 + 2 * cry] = -sin(0.);
		i0m[1 + 2 * cry] = cos(0.);
		i0m[0 + 2 * (cry + 1)] = -i0m[0 + 2 * cry];
		i0m[1 + 2 * (cry + 1)] = -i0m[1 + 2 * cry];
	}
	const int nx = s->pixpsax, ny = s->pixpsay;
	for (int isa = 0; isa < nsa; isa++) {
		const double* i0 = s->i0 + (size_t)isa * npix;
		for (int k = 0; k < npix * nmod; k++) A[k] = 0;
		for (int p = 0; p < npix; p++) {
			A[p + 0 * npix] = s->gx[(size_t)isa * npix + p];
			A[p + 1 * npix] = s->gy[(size_t)isa * npix + p];
			/* addvec twice with a NULL background image adds bkgrnd_res twice */
			A[p + 2 * npix] = i0[p] * kpx + bkgrnd_res + bkgrnd_res;
		}
		if (crx) { /* mki0sh(i0, kpx, 1, 0), lib/mtch.c:23-34 */
			for (int iy = 0; iy < ny; iy++)
				for (int ix = 0; ix < nx - 1; ix++) {
					A[(ix + 1) + iy * nx + crx * npix] = i0[ix + iy * nx] * kpx;
					A[ix + iy * nx + (crx + 1) * npix] = i0[(ix + 1) + iy * nx] * kpx;
				}
			for (int p = 0; p < npix; p++) {
				A[p + crx * npix] += bkgrnd_res;
				A[p + (crx + 1) * npix] += bkgrnd_res;
			}
		}
		if (cry) {
			for (int iy = 0; iy < ny - 1; iy++)
				for (int ix = 0; ix < nx; ix++) {
					A[ix + (iy + 1) * nx + cry * npix] = i0[ix + iy * nx] * kpy;
					A[ix + iy * nx + (cry + 1) * npix] = i0[ix + (iy + 1) * nx] * kpy;
				}
			for (int p = 0; p < npix; p++) {
				A[p + cry * npix] += bkgrnd_res;
				A[p + (cry + 1) * npix] += bkgrnd_res;
			}
		}
		for (int p = 0; p < npix; p++) {
			if (i0[p] < 0) wt[p] = 1. / rne2;
			else wt[p] = 1. / (rne2 + c->bkgrnd + i0[p]);
		}
		/* dpinv (math/blas.c:170-205): (A'WA)^-1 A'W with the SVD thresholds
		   1e-7 (absolute) and 1e-3 (relative to the previous kept value);
		   A'WA is symmetric, so its SVD is its eigen-decomposition. */
		for (int i = 0; i < nmod; i++)
			for (int j = 0; j < nmod; j++) {
				double v = 0;
				for (int p = 0; p < npix; p++) v += A[p + i * npix] * wt[p] * A[p + j * npix];
				cc[i + j * nmod] = v;
			}
		hsyev_jacobi(cc, nmod, ew, ev);
		int order_[7];
		for (int i = 0; i < nmod; i++) order_[i] = i;
		for (int i = 0; i < nmod; i++)
			for (int j = i + 1; j < nmod; j++)
				if (fabs(ew[order_[j]]) > fabs(ew[order_[i]])) {
					int tmp = order_[i];
					order_[i] = order_[j];
					order_[j] = tmp;
				}
		const double maxeig = fabs(ew[order_[0]]);
		const double thres10 = 1e-7 * maxeig;
		double thres20 = 1e-3 * maxeig;
		double sinv[7] = {0};
		for (int k = 0; k < nmod; k++) {
			const double sv = fabs(ew[order_[k]]);
			if (sv > thres10 && sv > thres20) {
				thres20 = sv * 1e-3;
				sinv[k] = 1. / ew[order_[k]];
			} else {
				break;
			}
		}
		for (int i = 0; i < nmod; i++)
			for (int j = 0; j < nmod; j++) {
				double v = 0;
				for (int k = 0; k < nmod; k++) v += ev[i + order_[k] * nmod] * sinv[k] * ev[j + order_[k] * nmod];
				inv[i + j * nmod] = v;
			}
		for (int i = 0; i < nmod; i++)
			for (int p = 0; p < npix; p++) {
				double v = 0;
				for (int k = 0; k < nmod; k++) v += inv[i + k * nmod] * A[p + k * npix] * wt[p];
				P[i + p * nmod] = v;
			}
		double* m = s->mtche + (size_t)isa * 2 * npix;
		for (int r = 0; r < 2; r++)
			for (int p = 0; p < npix; p++) {
				double v = 0;
				for (int k = 0; k < nmod; k++) v += i0m[r + 2 * k] * P[k + p * nmod];
				m[r + 2 * p] = v;
			}
		/* NEA (mtche * diag(1/wt) * mtche') and the rejection thresholds */
		double nea[4] = {0, 0, 0, 0};
		for (int r = 0; r < 2; r++)
			for (int q = 0; q < 2; q++)
				for (int p = 0; p < npix; p++) nea[r + 2 * q] += m[r + 2 * p] * (1. / wt[p]) * m[q + 2 * p];
		if (s->i0sum[isa] < i0thres || nea[0] > nea2thres || nea[3] > nea2thres) {
			for (int k = 0; k < 2 * npix; k++) m[k] = 0;
		}
	}
	free(A); free(wt); free(cc); free(ev); free(ew); free(inv); free(P);
	return 0;
}

int shwfs_setup_create(shwfs_setup** ps, const shwfs_setup_cfg* cfg) {
	if (!ps || !cfg) return SHWFS_EINVAL;
	*ps = NULL;
	shwfs_setup* s = calloc(1, sizeof(shwfs_setup));
	s->cfg = *cfg;
	int r;
	if (cfg->order <= 0 || !(cfg->dsa > 0) || !(cfg->dx > 0) || cfg->embfac <= 0 || cfg->pixpsa <= 0 ||
		!(cfg->wvl > 0) || !(cfg->pixtheta > 0)) {
		r = serr(s, "invalid configuration");
	} else if ((r = setup_geom(s)) == 0 && (r = setup_prep_phy(s)) == 0 && (r = setup_dtf(s)) == 0) {
		if (cfg->has_llt) {
			if (!((r = setup_etf(s)) == 0 && (r = setup_llt(s)) == 0)) goto out;
		}
		if (cfg->gradtype == SHWFS_GRAD_MF && (r = setup_seotf(s)) != 0) goto out;
		r = setup_mtch(s);
	}
out:
	*ps = s; /* returned also on failure so that the message can be read */
	return r;
}

void shwfs_setup_destroy(shwfs_setup* s) {
	if (!s) return;
	free(s->salocx); free(s->salocy); free(s->origx); free(s->origy); free(s->amp); free(s->saa);
	free(s->nominal); free(s->simap_idx); free(s->simap_wt); free(s->srot); free(s->srsa); free(s->etf);
	free(s->lltamp); free(s->mtche); free(s->i0sum); free(s->i0); free(s->gx); free(s->gy);
	free(s->sepsf); free(s->seotf);
	free(s);
}
const char* shwfs_setup_error(const shwfs_setup* s) { return s ? s->err : "null setup"; }
int shwfs_setup_nsa(const shwfs_setup* s) { return s->nsa; }
int shwfs_setup_nopd(const shwfs_setup* s) { return s->nopd; }
int shwfs_setup_notf(const shwfs_setup* s) { return s->notf; }
int shwfs_setup_npix(const shwfs_setup* s) { return s->npix; }
int shwfs_setup_llt_nx(const shwfs_setup* s) { return s->llt_nx; }
double shwfs_setup_dx(const shwfs_setup* s) { return s->dx; }
double shwfs_setup_areascale(const shwfs_setup* s) { return s->areascale; }
double shwfs_setup_dtheta(const shwfs_setup* s) { return s->dtheta; }
double shwfs_setup_i0sumsum(const shwfs_setup* s) { return s->i0sumsum; }
double shwfs_setup_saasum(const shwfs_setup* s) { return s->saasum; }

int shwfs_setup_get(const shwfs_setup* s, int what, double* out) {
	if (!s || !out) return SHWFS_EINVAL;
	const size_t nsa = s->nsa, n2 = (size_t)s->notf * s->notf, np = s->npix, no2 = (size_t)s->nopd * s->nopd;
	const double* src = NULL;
	size_t n = 0;
	switch (what) {
	case SHWFS_SETUP_SALOCX: src = s->salocx; n = nsa; break;
	case SHWFS_SETUP_SALOCY: src = s->salocy; n = nsa; break;
	case SHWFS_SETUP_ORIGX: src = s->origx; n = nsa; break;
	case SHWFS_SETUP_ORIGY: src = s->origy; n = nsa; break;
	case SHWFS_SETUP_AMP: src = s->amp; n = nsa * no2; break;
	case SHWFS_SETUP_SAA: src = s->saa; n = nsa; break;
	case SHWFS_SETUP_NOMINAL: src = s->nominal; n = n2; break;
	case SHWFS_SETUP_SIMAP_WT: src = s->simap_wt; n = np * 4; break;
	case SHWFS_SETUP_SROT: src = s->srot; n = nsa; break;
	case SHWFS_SETUP_SRSA: src = s->srsa; n = nsa; break;
	case SHWFS_SETUP_ETF: src = (const double*)s->etf; n = 2 * nsa * n2; break;
	case SHWFS_SETUP_LLTAMP: src = s->lltamp; n = (size_t)s->llt_nx * s->llt_nx; break;
	case SHWFS_SETUP_MTCHE: src = s->mtche; n = nsa * 2 * np; break;
	case SHWFS_SETUP_I0SUM: src = s->i0sum; n = nsa; break;
	case SHWFS_SETUP_I0: src = s->i0; n = nsa * np; break;
	case SHWFS_SETUP_GX: src = s->gx; n = nsa * np; break;
	case SHWFS_SETUP_GY: src = s->gy; n = nsa * np; break;
	case SHWFS_SETUP_SEPSF: src = s->sepsf; n = nsa * n2; break;
	case SHWFS_SETUP_SEOTF: src = (const double*)s->seotf; n = 2 * nsa * n2; break;
	default: return SHWFS_EINVAL;
	}
	if (!src) return SHWFS_EINVAL;
	memcpy(out, src, sizeof(double) * n);
	return 0;
}

int shwfs_setup_get_simap_idx(const shwfs_setup* s, int* out) {
	if (!s || !out || !s->simap_idx) return SHWFS_EINVAL;
	memcpy(out, s->simap_idx, sizeof(int) * s->npix * 4);
	return 0;
}

static void setup_desc(const shwfs_setup* s, shwfs_powfs_desc* pd);

int shwfs_setup_load(const shwfs_setup* s, shwfs_ctx* ctx, int* ipowfs) {
	if (!s || !ctx || !ipowfs) return SHWFS_EINVAL;
	const shwfs_setup_cfg* c = &s->cfg;
	shwfs_powfs_desc d;
	setup_desc(s, &d);
	int r = shwfs_powfs_add(ctx, &d, ipowfs);
	if (r) return r;
	if ((r = shwfs_powfs_set_geom(ctx, *ipowfs, s->origx, s->origy, s->amp, 1, s->saa))) return r;
	if ((r = shwfs_powfs_set_saasum(ctx, *ipowfs, s->saasum))) return r;
	if ((r = shwfs_powfs_set_simap(ctx, *ipowfs, s->simap_idx, s->simap_wt, 1))) return r;
	if (c->has_llt) {
		if ((r = shwfs_powfs_set_etf(ctx, *ipowfs, (const double*)s->etf, 0))) return r;
		if ((r = shwfs_powfs_set_lltamp(ctx, *ipowfs, s->lltamp))) return r;
	} else {
		if ((r = shwfs_powfs_set_nominal(ctx, *ipowfs, s->nominal, 1))) return r;
	}
	if (s->seotf && (r = shwfs_powfs_set_seotf(ctx, *ipowfs, (const double*)s->seotf))) return r;
	return 0;
}

int shwfs_setup_load_band(const shwfs_setup* s, shwfs_ctx* ctx, int ipowfs, double wvlwt, int* iband) {
	if (!s || !ctx || !iband) return SHWFS_EINVAL;
	shwfs_powfs_desc d;
	setup_desc(s, &d);
	int r = shwfs_powfs_add_band(ctx, ipowfs, &d, wvlwt, iband);
	if (r) return r;
	if ((r = shwfs_powfs_set_simap(ctx, *iband, s->simap_idx, s->simap_wt, 1))) return r;
	if (s->cfg.has_llt) return shwfs_powfs_set_etf(ctx, *iband, (const double*)s->etf, 0);
	return shwfs_powfs_set_nominal(ctx, *iband, s->nominal, 1);
}

static void setup_desc(const shwfs_setup* s, shwfs_powfs_desc* pd) {
	const shwfs_setup_cfg* c = &s->cfg;
	shwfs_powfs_desc d;
	memset(&d, 0, sizeof(d));
	d.nsa = s->nsa;
	d.nopd = s->nopd;
	d.embfac = c->embfac;
	d.notf = s->notf;
	d.pixpsax = s->pixpsax;
	d.pixpsay = s->pixpsay;
	d.pixthetax = d.pixthetay = c->pixtheta;
	d.wvl = c->wvl;
	d.dsa = c->dsa;
	d.dx = s->dx;
	d.areascale = s->areascale;
	d.hs = c->hs;
	d.has_etf = c->has_llt;
	d.has_llt = c->has_llt;
	d.llt_nx = s->llt_nx;
	d.llt_ox = c->llt_ox;
	d.llt_oy = c->llt_oy;
	d.llt_origx = d.llt_origy = s->llt_orig;
	d.gradtype = c->gradtype;
	d.sigmatch = c->sigmatch;
	d.cogthres = c->cogthres;
	d.cogoff = c->cogoff;
	d.rne = c->rne;
	d.bkgrnd = c->bkgrnd;
	d.bkgrndc = c->bkgrnd * c->bkgrndc;
	d.saat = c->saat;
	d.sigtot_cog = c->siglev;
	*pd = d;
}

int shwfs_setup_load_wfs(const shwfs_setup* s, shwfs_ctx* ctx, int iwfs) {
	if (!s || !ctx) return SHWFS_EINVAL;
	return shwfs_wfs_set_mtche(ctx, iwfs, s->mtche, s->i0sum, s->i0sumsum);
}

/* ---- screens: lib/turbulence.c:70-168 and :436-478 ---- */
int shwfs_screens_vonkarman(double* const* out, int nlayer, long nx, long ny, double dx, double r0, double L0,
	const double* wt, uint32_t seed) {
	if (!out || nlayer <= 0 || nx < 2 || ny < 2 || !(dx > 0) || !(r0 > 0) || !wt) return SHWFS_EINVAL;
	hrand r;
	hrand_seed(&r, seed);
	const double slope = -11. / 3. * 0.5 / 2.;
	const double strength = 0.0229 * pow(r0, -5. / 3.) * pow((0.5e-6) / (2. * M_PI), 2);
	const double dfx = 1. / (nx * dx), dfy = 1. / (ny * dx);
	const double zerofreq2 = L0 == 0 ? 0 : pow(L0, -2);
	const double scrnstr = pow(strength * (dfx * dfy), 0.5);
	const long nx2 = nx / 2, ny2 = ny / 2;
	double* psd = malloc(sizeof(double) * nx * ny);
	for (long iy = 0; iy < ny; iy++) {
		const double r2y = pow((iy < ny2 ? iy : iy - ny) * dfy, 2);
		for (long ix = 0; ix < nx; ix++) {
			const double r2 = pow((ix < nx2 ? ix : ix - nx) * dfx, 2) + r2y;
			psd[ix + iy * nx] = pow(r2 + zerofreq2, slope) * scrnstr;
		}
	}
	psd[0] = 0;
	double* p1 = malloc(sizeof(double) * nx * ny);
	double* p2 = malloc(sizeof(double) * nx * ny);
	for (int il = 0; il < nlayer; il += 2) {
		for (long i = 0; i < nx * ny; i++) {
			p1[i] = hrand_normal(&r) * psd[i];
			p2[i] = hrand_normal(&r) * psd[i];
		}
		hfft2_split(p1, p2, nx, ny);
		const double s1 = sqrt(wt[il]);
		for (long i = 0; i < nx * ny; i++) out[il][i] = p1[i] * s1;
		if (il + 1 < nlayer) {
			const double s2 = sqrt(wt[il + 1]);
			for (long i = 0; i < nx * ny; i++) out[il + 1][i] = p2[i] * s2;
		}
	}
	free(psd);
	free(p1);
	free(p2);
	return 0;
}

/* ---- science aperture: maos/aper.c:45-110 for an annulus ---- */

/* X(circle) (math/matmath.c:476-516) on an nx x ny map of spacing dx with
   centre (cx, cy) in map coordinates, val 1: the bilinear-weighted coverage
   of each point, kept as the mask (coverage > 1e-15) create_metapupil uses. */
static int circle_mask_pt(int ix, int iy, double cx, double cy, double dx, double r) {
	const int nres = 10;
	const double res = 2. / nres, res2 = res * res, resm = (nres - 1) * 0.5;
	const double r2 = r * r;
	const double r2l = r > 1.5 ? ((r - 1.5) * (r - 1.5)) : 0;
	const double r2u = (r + 2.5) * (r + 2.5);
	const double r2y = (iy * dx - cy) * (iy * dx - cy);
	const double r2r = (ix * dx - cx) * (ix * dx - cx) + r2y;
	double v = 0;
	if (r2r < r2l) {
		v = 1;
	} else if (r2r < r2u) {
		double tot = 0.;
		for (int jy = 0; jy < nres; jy++) {
			const double iiy = iy + (jy - resm) * res;
			const double rr2y = (iiy * dx - cy) * (iiy * dx - cy);
			const double wty = 1. - fabs(iy - iiy);
			for (int jx = 0; jx < nres; jx++) {
				const double iix = ix + (jx - resm) * res;
				const double rr2r = (iix * dx - cx) * (iix * dx - cx) + rr2y;
				const double wtx = 1. - fabs(ix - iix);
				if (rr2r < r2) tot += res2 * wty * wtx;
			}
		}
		v = tot;
	}
	return v > 1.e-15;
}

int shwfs_aper_build(double D, double Din, double dx, long* nloc, double* locx, double* locy, double* amp) {
	if (!nloc || !(D > 0) || !(dx > 0) || Din < 0 || Din >= D) return SHWFS_EINVAL;
	const double R = D / 2, guard = dx;
	// create_metapupil (math/map.c:144-182) with ht0 = 0, offset 0, no padding
	const double minx = -R - guard, maxx = R + guard;
	const double ox = floor(minx / dx) * dx;
	const long nx = (long)ceil((maxx - ox) / dx) + 1;
	const double oy = floor(minx / dx) * dx;
	const long ny = (long)ceil((maxx - oy) / dx) + 1;
	if (nx > 100000) return SHWFS_EINVAL;
	const long cap = locx ? *nloc : 0;
	double* row = (double*)malloc(sizeof(double) * nx);
	double* ax = locx ? (double*)malloc(sizeof(double) * (cap > 0 ? cap : 1)) : NULL;
	if (!row || (locx && !ax)) {
		free(row);
		free(ax);
		return SHWFS_ENOMEM;
	}
	long count = 0;
	for (long iy = 0; iy < ny; iy++) {
		// loc_from_map: the row from its first to its last masked point
		long i0 = -1, i1 = -1;
		for (long ix = 0; ix < nx && i0 < 0; ix++)
			if (circle_mask_pt((int)ix, (int)iy, -ox, -oy, dx, R)) i0 = ix;
		for (long ix = nx - 1; ix > -1 && i1 < 0; ix--)
			if (circle_mask_pt((int)ix, (int)iy, -ox, -oy, dx, R)) i1 = ix;
		if (i0 < 0) continue;
		// mkamp: loc_circle_add of the annulus; loc_reduce (cont = 1) drops
		// the row's leading and trailing points below EPS
		long j0 = -1, j1 = -1;
		for (long ix = i0; ix <= i1; ix++) {
			const double x = ix * dx + ox, y = iy * dx + oy;
			double a = circle_add_pt(x, y, dx, R, 1);
			if (Din > 0) a += circle_add_pt(x, y, dx, Din * 0.5, -1);
			row[ix] = a;
			if (a >= 1.e-15) {
				if (j0 < 0) j0 = ix;
				j1 = ix;
			}
		}
		if (j0 < 0) continue;
		for (long ix = j0; ix <= j1; ix++, count++) {
			if (!locx) continue;
			if (count >= cap) {
				free(row);
				free(ax);
				return SHWFS_EINVAL;
			}
			locx[count] = ix * dx + ox;
			locy[count] = iy * dx + oy;
			ax[count] = row[ix];
		}
	}
	if (locx) {
		double sum = 0;  // dnormalize_sum: scale by 1 / (sequential sum)
		for (long i = 0; i < count; i++) sum += ax[i];
		const double w = 1. / sum;
		for (long i = 0; i < count; i++) amp[i] = ax[i] * w;
	}
	free(row);
	free(ax);
	*nloc = count;
	return 0;
}
