/* Host-side numerics used by the setup producers: double-precision FFT,
   the reference's random streams, small dense linear algebra. */
#ifndef SHWFS_HMATH_H
#define SHWFS_HMATH_H
#include <complex.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex hcplx;

/* In-place 2-D DFT of an nx*ny column-major (x fastest) array, FFTW sign
   convention (dir=-1: exp(-2*pi*i...), dir=+1: exp(+...)), unnormalised. */
void hfft2(hcplx* a, long nx, long ny, int dir);
/* 2-D forward DFT of the complex array re + i*im held as two real arrays
   (the split form the reference uses to make two screens per transform). */
void hfft2_split(double* re, double* im, long nx, long ny);
/* fftshift of an nx*ny complex array (swap quadrants). */
void hfftshift(hcplx* a, long nx, long ny);

/* Mersenne twister in the reference's seeding and draw order
   (math/random.c:84-181, math/random.h:158-167). */
typedef struct hrand {
	uint32_t mt[624];
	int idx;
} hrand;
void hrand_seed(hrand* r, uint32_t seed);
uint32_t hrand_u32(hrand* r);
double hrand_u01(hrand* r);       /* [0,1), 32-bit resolution */
double hrand_normal(hrand* r);    /* ziggurat of math/random.c:211-315 */
long hrand_poisson(hrand* r, double mean); /* math/random.c:186-209 */

/* Symmetric eigen-decomposition by cyclic Jacobi rotations: a (n x n,
   column-major) is overwritten, w receives eigenvalues, v eigenvectors
   (columns).  Used for the small normal matrix of the matched filter. */
void hsyev_jacobi(double* a, int n, double* w, double* v);

#ifdef __cplusplus
}
#endif
#endif
