/*
 * Implementation of the FFTW3 stand-in declared in fftw3.h.  Test
 * infrastructure for the oracle: it lets the reference's own math/fft.c (and
 * through it wfsints, mkdtf, mketf, gensei and the screen generator) be
 * compiled and run here without libfftw3.
 *
 * Algorithm: the discrete Fourier transform as FFTW defines it
 *   Y[k] = sum_j X[j] exp(sign * 2*pi*i * j*k / n),   no scaling,
 * evaluated with an iterative radix-2 Cooley-Tukey FFT for power-of-two n and
 * a direct O(n^2) sum otherwise.  Twiddles are computed directly from
 * cos/sin of the reduced angle (no recurrences) so round-off stays near the
 * FFTW level (~1e-16 relative).  Multi-dimensional and batched plans are
 * composed of strided 1-D transforms.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

enum { K_DFT=0, K_SPLIT=1, K_R2R=2 };

/* One group of strided 1-D transforms: for h in [0,howmany), transform the
   length-n sequence at base + h*dist with element stride `stride`. */
typedef struct {
	int n, stride, dist, howmany;
} pass_t;

struct fftw_plan_s {
	int kind;
	int sign;
	int npass;
	pass_t pass[4];
	double* re; /* interleaved data (K_DFT) or split real part */
	double* im; /* split imaginary part (K_SPLIT) */
	int r2r_kind;
	int n_r2r;
};

static int is_pow2(int n){ return n>0 && (n&(n-1))==0; }

/* In-place complex transform of a contiguous buffer xr/xi of length n. */
static void dft_contig(double* xr, double* xi, int n, int sign){
	if(n<=1) return;
	if(is_pow2(n)){
		/* bit reversal */
		for(int i=1, j=0; i<n; i++){
			int bit=n>>1;
			for(; j&bit; bit>>=1) j^=bit;
			j^=bit;
			if(i<j){
				double t=xr[i]; xr[i]=xr[j]; xr[j]=t;
				t=xi[i]; xi[i]=xi[j]; xi[j]=t;
			}
		}
		for(int len=2; len<=n; len<<=1){
			int half=len>>1;
			for(int k=0; k<half; k++){
				double ang=sign*2.0*M_PI*(double)k/(double)len;
				double wr=cos(ang), wi=sin(ang);
				for(int s=0; s<n; s+=len){
					int a=s+k, b=a+half;
					double tr=xr[b]*wr-xi[b]*wi;
					double ti=xr[b]*wi+xi[b]*wr;
					xr[b]=xr[a]-tr; xi[b]=xi[a]-ti;
					xr[a]+=tr; xi[a]+=ti;
				}
			}
		}
	} else{
		double* yr=malloc(sizeof(double)*n*2);
		double* yi=yr+n;
		for(int k=0; k<n; k++){
			double sr=0, si=0;
			for(int j=0; j<n; j++){
				long m=((long)j*k)%n;
				double ang=sign*2.0*M_PI*(double)m/(double)n;
				double c=cos(ang), s=sin(ang);
				sr+=xr[j]*c-xi[j]*s;
				si+=xr[j]*s+xi[j]*c;
			}
			yr[k]=sr; yi[k]=si;
		}
		memcpy(xr, yr, sizeof(double)*n);
		memcpy(xi, yi, sizeof(double)*n);
		free(yr);
	}
}

static void run_pass_interleaved(double* base, const pass_t* p, int sign){
	double* xr=malloc(sizeof(double)*p->n*2);
	double* xi=xr+p->n;
	for(int h=0; h<p->howmany; h++){
		double* b=base+2L*(long)h*p->dist;
		for(int j=0; j<p->n; j++){
			xr[j]=b[2L*j*p->stride];
			xi[j]=b[2L*j*p->stride+1];
		}
		dft_contig(xr, xi, p->n, sign);
		for(int j=0; j<p->n; j++){
			b[2L*j*p->stride]=xr[j];
			b[2L*j*p->stride+1]=xi[j];
		}
	}
	free(xr);
}

static void run_pass_split(double* re, double* im, const pass_t* p, int sign){
	double* xr=malloc(sizeof(double)*p->n*2);
	double* xi=xr+p->n;
	for(int h=0; h<p->howmany; h++){
		long off=(long)h*p->dist;
		for(int j=0; j<p->n; j++){
			xr[j]=re[off+(long)j*p->stride];
			xi[j]=im[off+(long)j*p->stride];
		}
		dft_contig(xr, xi, p->n, sign);
		for(int j=0; j<p->n; j++){
			re[off+(long)j*p->stride]=xr[j];
			im[off+(long)j*p->stride]=xi[j];
		}
	}
	free(xr);
}

static fftw_plan plan_alloc(int kind, int sign){
	fftw_plan p=calloc(1, sizeof(struct fftw_plan_s));
	p->kind=kind;
	p->sign=sign;
	return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags){
	(void)flags;
	if(in!=out) return NULL; /* the reference only plans in-place transforms */
	fftw_plan p=plan_alloc(K_DFT, sign);
	p->re=(double*)in;
	p->npass=1;
	p->pass[0]=(pass_t){n, 1, 0, 1};
	return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags){
	(void)flags;
	if(in!=out) return NULL;
	fftw_plan p=plan_alloc(K_DFT, sign);
	p->re=(double*)in;
	p->npass=2;
	p->pass[0]=(pass_t){n1, 1, n1, n0}; /* contiguous rows */
	p->pass[1]=(pass_t){n0, n1, 1, n1}; /* strided columns */
	return p;
}

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
	fftw_complex* in, const int* inembed, int istride, int idist,
	fftw_complex* out, const int* onembed, int ostride, int odist,
	int sign, unsigned flags){
	(void)inembed; (void)onembed; (void)flags;
	if(rank!=1||in!=out||istride!=ostride||idist!=odist) return NULL;
	fftw_plan p=plan_alloc(K_DFT, sign);
	p->re=(double*)in;
	p->npass=1;
	p->pass[0]=(pass_t){n[0], istride, idist, howmany};
	return p;
}

fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim* dims,
	int howmany_rank, const fftw_iodim* howmany_dims,
	double* ri, double* ii, double* ro, double* io, unsigned flags){
	(void)flags;
	if(ri!=ro||ii!=io||rank<1||rank>2||howmany_rank!=1||howmany_dims[0].n!=1) return NULL;
	/* FFTW's split-array interface always computes the forward transform. */
	fftw_plan p=plan_alloc(K_SPLIT, FFTW_FORWARD);
	p->re=ri;
	p->im=ii;
	p->npass=rank;
	if(rank==1){
		p->pass[0]=(pass_t){dims[0].n, dims[0].is, 0, 1};
	} else{
		/* dims[0] and dims[1] are independent axes; transform each over the
		   other's full extent. */
		p->pass[0]=(pass_t){dims[0].n, dims[0].is, dims[1].is, dims[1].n};
		p->pass[1]=(pass_t){dims[1].n, dims[1].is, dims[0].is, dims[0].n};
	}
	return p;
}

fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind, unsigned flags){
	(void)flags;
	if(in!=out) return NULL;
	fftw_plan p=plan_alloc(K_R2R, 0);
	p->re=in;
	p->r2r_kind=kind;
	p->n_r2r=n;
	return p;
}

/* FFTW halfcomplex layout: r0, r1..r_{n/2}, i_{(n+1)/2-1}..i1. */
static void run_r2r(double* x, int n, int kind){
	double* xr=calloc(2*(size_t)n, sizeof(double));
	double* xi=xr+n;
	if(kind==FFTW_R2HC){
		for(int j=0; j<n; j++) xr[j]=x[j];
		dft_contig(xr, xi, n, FFTW_FORWARD);
		x[0]=xr[0];
		for(int k=1; k<=n/2; k++) x[k]=xr[k];
		for(int k=1; k<(n+1)/2; k++) x[n-k]=xi[k];
	} else{
		xr[0]=x[0];
		for(int k=1; k<=n/2; k++) xr[k]=x[k];
		for(int k=1; k<(n+1)/2; k++) xi[k]=x[n-k];
		for(int k=1; k<(n+1)/2; k++){ xr[n-k]=xr[k]; xi[n-k]=-xi[k]; }
		dft_contig(xr, xi, n, FFTW_BACKWARD);
		for(int j=0; j<n; j++) x[j]=xr[j];
	}
	free(xr);
}

void fftw_execute(const fftw_plan p){
	if(!p) return;
	switch(p->kind){
	case K_DFT:
		for(int i=0; i<p->npass; i++) run_pass_interleaved(p->re, &p->pass[i], p->sign);
		break;
	case K_SPLIT:
		for(int i=0; i<p->npass; i++) run_pass_split(p->re, p->im, &p->pass[i], p->sign);
		break;
	case K_R2R:
		run_r2r(p->re, p->n_r2r, p->r2r_kind);
		break;
	}
}

void fftw_destroy_plan(fftw_plan p){ free(p); }
int fftw_import_wisdom_from_file(FILE* f){ (void)f; return 0; }
void fftw_export_wisdom_to_file(FILE* f){ (void)f; }
int fftw_init_threads(void){ return 1; }
void fftw_plan_with_nthreads(int nthreads){ (void)nthreads; }
