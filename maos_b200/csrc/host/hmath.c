/* Host numerics for the setup producers (see hmath.h). */
#include "hmath.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------- FFT ---------------- */
static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place transform of a contiguous sequence (radix-2 for powers of two,
   direct sum otherwise).  Twiddles from cos/sin of the exact angle. */
static void fft1(hcplx* x, long n, int dir, hcplx* tmp) {
	if (n <= 1) return;
	if (is_pow2(n)) {
		for (long i = 1, j = 0; i < n; i++) {
			long bit = n >> 1;
			for (; j & bit; bit >>= 1) j ^= bit;
			j ^= bit;
			if (i < j) {
				hcplx t = x[i];
				x[i] = x[j];
				x[j] = t;
			}
		}
		for (long len = 2; len <= n; len <<= 1) {
			const long half = len >> 1;
			for (long k = 0; k < half; k++) {
				const double ang = dir * 2.0 * M_PI * (double)k / (double)len;
				const hcplx w = cos(ang) + I * sin(ang);
				for (long s = 0; s < n; s += len) {
					const hcplx u = x[s + k], v = x[s + k + half] * w;
					x[s + k] = u + v;
					x[s + k + half] = u - v;
				}
			}
		}
	} else {
		for (long k = 0; k < n; k++) {
			hcplx acc = 0;
			for (long j = 0; j < n; j++) {
				const long m = (j * k) % n;
				const double ang = dir * 2.0 * M_PI * (double)m / (double)n;
				acc += x[j] * (cos(ang) + I * sin(ang));
			}
			tmp[k] = acc;
		}
		memcpy(x, tmp, sizeof(hcplx) * n);
	}
}

void hfft2(hcplx* a, long nx, long ny, int dir) {
	const long nmax = nx > ny ? nx : ny;
	hcplx* buf = malloc(sizeof(hcplx) * nmax * 2);
	hcplx* tmp = buf + nmax;
	for (long iy = 0; iy < ny; iy++) fft1(a + iy * nx, nx, dir, tmp);
	for (long ix = 0; ix < nx; ix++) {
		for (long iy = 0; iy < ny; iy++) buf[iy] = a[ix + iy * nx];
		fft1(buf, ny, dir, tmp);
		for (long iy = 0; iy < ny; iy++) a[ix + iy * nx] = buf[iy];
	}
	free(buf);
}

void hfft2_split(double* re, double* im, long nx, long ny) {
	hcplx* a = malloc(sizeof(hcplx) * nx * ny);
	for (long i = 0; i < nx * ny; i++) a[i] = re[i] + I * im[i];
	hfft2(a, nx, ny, -1);
	for (long i = 0; i < nx * ny; i++) {
		re[i] = creal(a[i]);
		im[i] = cimag(a[i]);
	}
	free(a);
}

void hfftshift(hcplx* a, long nx, long ny) {
	const long nx2 = nx / 2, ny2 = ny / 2;
	hcplx* t = malloc(sizeof(hcplx) * nx * ny);
	for (long iy = 0; iy < ny; iy++)
		for (long ix = 0; ix < nx; ix++) t[((ix + nx2) % nx) + ((iy + ny2) % ny) * nx] = a[ix + iy * nx];
	memcpy(a, t, sizeof(hcplx) * nx * ny);
	free(t);
}

/* ---------------- random streams ---------------- */
/* Seeding: mt[0] = ~seed (4357 if that is 0), mt[j] = 69069*mt[j-1]; the
   state is twisted before the first draw (math/random.c:143-181). */
static void hrand_twist(hrand* r) {
	uint32_t* mt = r->mt;
	for (int i = 0; i < 624; i++) {
		const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
		mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
	}
	r->idx = 0;
}
void hrand_seed(hrand* r, uint32_t seed) {
	uint32_t s = ~seed;
	if (s == 0) s = 4357u;
	r->mt[0] = s;
	for (int j = 1; j < 624; j++) r->mt[j] = 69069u * r->mt[j - 1];
	hrand_twist(r);
}
uint32_t hrand_u32(hrand* r) {
	if (r->idx >= 624) hrand_twist(r);
	uint32_t v = r->mt[r->idx++];
	v ^= v >> 11;
	v ^= (v << 7) & 0x9d2c5680u;
	v ^= (v << 15) & 0xefc60000u;
	v ^= v >> 18;
	return v;
}
double hrand_u01(hrand* r) { return hrand_u32(r) * (1.0 / 4294967296.0); }

/* Ziggurat tables (256 levels) built as in math/random.c:227-281. */
#define ZLEV 256
static double zx[ZLEV], zy[ZLEV], zk[ZLEV], zw[ZLEV], zx1, zx11, zv;
static int z_ready = 0;
static double zf(double x) { return exp(-x * x * 0.5); }
static double zfinv(double y) { return sqrt(-2. * log(y)); }
static double ztry(double r) {
	zv = r * zf(r) + exp(-0.5 * r * r) / r;
	zx[ZLEV - 1] = r;
	for (int i = ZLEV - 1; i > 1; --i) zx[i - 1] = zfinv(zv / zx[i] + zf(zx[i]));
	return zx[1] * (1 - zf(zx[1])) / zv;
}
static void z_init(void) {
	double a = 0, b = 10, aa, bb, r;
	do {
		aa = a;
		bb = b;
		r = .5 * (a + b);
		const double q = ztry(r);
		if (q > 1) b = r;
		else a = r;
	} while (aa < r && r < bb);
	zx[0] = 0;
	zx1 = r;
	zx11 = 1. / zx1;
	for (int i = 0; i < ZLEV; i++) zy[i] = zf(zx[i]);
	for (int i = 0; i < ZLEV - 1; i++) zk[i] = zx[i] / zx[i + 1];
	zk[ZLEV - 1] = zx1 * zf(zx1) / zv;
	for (int i = 0; i < ZLEV - 1; i++) zw[i] = zx[i + 1];
	zw[ZLEV - 1] = zv / zf(zx1);
	z_ready = 1;
}
double hrand_normal(hrand* r) {
	if (!z_ready) z_init();
	double x;
	for (;;) {
		const double U = 2 * hrand_u01(r) - 1;
		const uint32_t l = hrand_u32(r);
		const int i = (int)(l & (ZLEV - 1));
		x = U * zw[i];
		if (fabs(U) < zk[i]) break;
		if (i == ZLEV - 1) {
			double x0, y;
			do {
				x0 = log(hrand_u01(r)) * zx11;
				y = -log(hrand_u01(r));
			} while (y + y < x0 * x0);
			x = x > 0 ? (zx1 - x0) : (x0 - zx1);
			break;
		} else {
			const double y = zy[i + 1] + (zy[i] - zy[i + 1]) * hrand_u01(r);
			if (y < zf(x)) break;
		}
	}
	return x;
}
long hrand_poisson(hrand* r, double xm) {
	long x = 0;
	if (xm > 200) {
		x = (long)round(xm + hrand_normal(r) * sqrt(xm));
	} else {
		while (xm > 0) {
			const double xmu = xm > 12 ? 12 : xm;
			xm -= xmu;
			const double g = exp(-xmu);
			long xu = -1;
			double t = 1;
			while (t > g) {
				xu++;
				t *= hrand_u01(r);
			}
			x += xu;
		}
	}
	return x;
}

/* ---------------- Jacobi eigen-decomposition ---------------- */
void hsyev_jacobi(double* a, int n, double* w, double* v) {
	for (int i = 0; i < n * n; i++) v[i] = 0;
	for (int i = 0; i < n; i++) v[i + i * n] = 1;
	for (int sweep = 0; sweep < 100; sweep++) {
		double off = 0, diag = 0;
		for (int p = 0; p < n; p++) {
			diag += a[p + p * n] * a[p + p * n];
			for (int q = p + 1; q < n; q++) off += a[p + q * n] * a[p + q * n];
		}
		if (off <= 1e-30 * diag || off == 0) break;
		for (int p = 0; p < n - 1; p++) {
			for (int q = p + 1; q < n; q++) {
				const double apq = a[p + q * n];
				if (apq == 0) continue;
				const double theta = (a[q + q * n] - a[p + p * n]) / (2 * apq);
				const double t = (theta >= 0 ? 1 : -1) / (fabs(theta) + sqrt(1 + theta * theta));
				const double c = 1 / sqrt(1 + t * t), s = t * c;
				for (int k = 0; k < n; k++) {
					const double akp = a[k + p * n], akq = a[k + q * n];
					a[k + p * n] = c * akp - s * akq;
					a[k + q * n] = s * akp + c * akq;
				}
				for (int k = 0; k < n; k++) {
					const double apk = a[p + k * n], aqk = a[q + k * n];
					a[p + k * n] = c * apk - s * aqk;
					a[q + k * n] = s * apk + c * aqk;
				}
				for (int k = 0; k < n; k++) {
					const double vkp = v[k + p * n], vkq = v[k + q * n];
					v[k + p * n] = c * vkp - s * vkq;
					v[k + q * n] = s * vkp + c * vkq;
				}
			}
		}
	}
	for (int i = 0; i < n; i++) w[i] = a[i + i * n];
}
