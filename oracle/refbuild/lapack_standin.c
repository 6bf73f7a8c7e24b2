/*
 * Stand-ins for the few BLAS/LAPACK entry points that the reference's own C
 * reaches on the Shack-Hartmann path when it is compiled as the test oracle
 * (oracle/_ref).  The reference links a system BLAS/LAPACK (OpenBLAS or MKL);
 * none is installed here.  Test infrastructure only.
 *
 *  - dgemm_/zgemm_: C = alpha*op(A)*op(B) + beta*C, column-major, as the
 *    reference BLAS defines it (plain triple loop).
 *  - dgesvd_/dgesdd_ with job 'S': thin SVD by one-sided (Hestenes) Jacobi
 *    rotations, singular values sorted in decreasing order.  The reference
 *    uses it only to invert the small (<=7x7) normal matrix of the matched
 *    filter (lib/mtch.c -> math/blas.c dpinv -> svd_pow2).
 *  - dpotrf_/dposv_/dgesv_: Cholesky and LU solves (textbook algorithms),
 *    reached by the PSD fit of the screen known-answer test.
 *  - every other routine the reference declares aborts with a message, so an
 *    unexpected call cannot pass silently.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int is_t(const char* c){ return *c=='T'||*c=='t'||*c=='C'||*c=='c'; }
static int is_c(const char* c){ return *c=='C'||*c=='c'; }

void dgemm_(const char* ta, const char* tb, const ptrdiff_t* m, const ptrdiff_t* n, const ptrdiff_t* k,
	const double* alpha, const double* A, const ptrdiff_t* lda, const double* B, const ptrdiff_t* ldb,
	const double* beta, double* C, const ptrdiff_t* ldc){
	const int tA=is_t(ta), tB=is_t(tb);
	for(ptrdiff_t j=0; j<*n; j++){
		for(ptrdiff_t i=0; i<*m; i++){
			double s=0;
			for(ptrdiff_t l=0; l<*k; l++){
				double a=tA?A[l+i*(*lda)]:A[i+l*(*lda)];
				double b=tB?B[j+l*(*ldb)]:B[l+j*(*ldb)];
				s+=a*b;
			}
			double* c=&C[i+j*(*ldc)];
			*c=(*beta==0?0:(*beta)*(*c))+(*alpha)*s;
		}
	}
}

void zgemm_(const char* ta, const char* tb, const ptrdiff_t* m, const ptrdiff_t* n, const ptrdiff_t* k,
	const double complex* alpha, const double complex* A, const ptrdiff_t* lda,
	const double complex* B, const ptrdiff_t* ldb,
	const double complex* beta, double complex* C, const ptrdiff_t* ldc){
	const int tA=is_t(ta), tB=is_t(tb), cA=is_c(ta), cB=is_c(tb);
	for(ptrdiff_t j=0; j<*n; j++){
		for(ptrdiff_t i=0; i<*m; i++){
			double complex s=0;
			for(ptrdiff_t l=0; l<*k; l++){
				double complex a=tA?A[l+i*(*lda)]:A[i+l*(*lda)];
				double complex b=tB?B[j+l*(*ldb)]:B[l+j*(*ldb)];
				if(cA) a=conj(a);
				if(cB) b=conj(b);
				s+=a*b;
			}
			double complex* c=&C[i+j*(*ldc)];
			*c=(*beta==0?0:(*beta)*(*c))+(*alpha)*s;
		}
	}
}

/* Thin SVD of the m x n column-major matrix a (m>=n): a = U diag(s) V'.
   On return u is m x n, s has n entries (descending), vt is n x n. */
static int jacobi_svd_tall(ptrdiff_t m, ptrdiff_t n, const double* a, ptrdiff_t lda,
	double* s, double* u, ptrdiff_t ldu, double* vt, ptrdiff_t ldvt){
	double* w=malloc(sizeof(double)*m*n);
	double* v=calloc((size_t)(n*n), sizeof(double));
	for(ptrdiff_t j=0; j<n; j++){
		memcpy(w+j*m, a+j*lda, sizeof(double)*m);
		v[j+j*n]=1;
	}
	for(int sweep=0; sweep<100; sweep++){
		double off=0;
		for(ptrdiff_t p=0; p<n-1; p++){
			for(ptrdiff_t q=p+1; q<n; q++){
				double alpha=0, beta=0, gamma=0;
				for(ptrdiff_t i=0; i<m; i++){
					alpha+=w[i+p*m]*w[i+p*m];
					beta+=w[i+q*m]*w[i+q*m];
					gamma+=w[i+p*m]*w[i+q*m];
				}
				if(gamma==0) continue;
				double r=fabs(gamma)/sqrt(alpha*beta);
				if(r>off) off=r;
				if(r<1e-15) continue;
				double zeta=(beta-alpha)/(2*gamma);
				double t=(zeta>=0?1:-1)/(fabs(zeta)+sqrt(1+zeta*zeta));
				double c=1/sqrt(1+t*t), sn=c*t;
				for(ptrdiff_t i=0; i<m; i++){
					double xp=w[i+p*m], xq=w[i+q*m];
					w[i+p*m]=c*xp-sn*xq;
					w[i+q*m]=sn*xp+c*xq;
				}
				for(ptrdiff_t i=0; i<n; i++){
					double xp=v[i+p*n], xq=v[i+q*n];
					v[i+p*n]=c*xp-sn*xq;
					v[i+q*n]=sn*xp+c*xq;
				}
			}
		}
		if(off<1e-15) break;
	}
	/* singular values are column norms; sort descending */
	ptrdiff_t* idx=malloc(sizeof(ptrdiff_t)*n);
	double* sv=malloc(sizeof(double)*n);
	for(ptrdiff_t j=0; j<n; j++){
		double t=0;
		for(ptrdiff_t i=0; i<m; i++) t+=w[i+j*m]*w[i+j*m];
		sv[j]=sqrt(t);
		idx[j]=j;
	}
	for(ptrdiff_t i=0; i<n; i++){
		for(ptrdiff_t j=i+1; j<n; j++){
			if(sv[idx[j]]>sv[idx[i]]){ ptrdiff_t t=idx[i]; idx[i]=idx[j]; idx[j]=t; }
		}
	}
	for(ptrdiff_t k=0; k<n; k++){
		ptrdiff_t j=idx[k];
		s[k]=sv[j];
		for(ptrdiff_t i=0; i<m; i++){
			u[i+k*ldu]=sv[j]>0?w[i+j*m]/sv[j]:(i==k?1:0);
		}
		for(ptrdiff_t i=0; i<n; i++){
			vt[k+i*ldvt]=v[i+j*n];
		}
	}
	free(idx); free(sv); free(w); free(v);
	return 0;
}

static void svd_thin(ptrdiff_t m, ptrdiff_t n, double* a, ptrdiff_t lda, double* s,
	double* u, ptrdiff_t ldu, double* vt, ptrdiff_t ldvt){
	if(m>=n){
		jacobi_svd_tall(m, n, a, lda, s, u, ldu, vt, ldvt);
	} else{
		/* a' = V diag(s) U' : run on the transpose and swap the factors */
		double* at=malloc(sizeof(double)*m*n);
		for(ptrdiff_t i=0; i<m; i++) for(ptrdiff_t j=0; j<n; j++) at[j+i*n]=a[i+j*lda];
		double* ut=malloc(sizeof(double)*n*m);
		double* vtt=malloc(sizeof(double)*m*m);
		jacobi_svd_tall(n, m, at, n, s, ut, n, vtt, m);
		/* u (m x m) = vtt', vt (m x n) = ut' */
		for(ptrdiff_t i=0; i<m; i++) for(ptrdiff_t k=0; k<m; k++) u[i+k*ldu]=vtt[k+i*m];
		for(ptrdiff_t k=0; k<m; k++) for(ptrdiff_t j=0; j<n; j++) vt[k+j*ldvt]=ut[j+k*n];
		free(at); free(ut); free(vtt);
	}
}

void dgesvd_(const char* jobu, const char* jobvt, ptrdiff_t* m, ptrdiff_t* n, double* a,
	ptrdiff_t* lda, double* s, double* u, ptrdiff_t* ldu, double* vt, ptrdiff_t* ldvt,
	double* work, ptrdiff_t* lwork, ptrdiff_t* info){
	(void)jobu; (void)jobvt;
	*info=0;
	if(*lwork==-1){ work[0]=1; return; }
	svd_thin(*m, *n, a, *lda, s, u, *ldu, vt, *ldvt);
}

void dgesdd_(const char* jobz, ptrdiff_t* m, ptrdiff_t* n, double* a, ptrdiff_t* lda,
	double* s, double* u, ptrdiff_t* ldu, double* vt, ptrdiff_t* ldvt,
	double* work, ptrdiff_t* lwork, ptrdiff_t* iwork, ptrdiff_t* info){
	(void)jobz; (void)iwork;
	*info=0;
	if(*lwork==-1){ work[0]=1; return; }
	svd_thin(*m, *n, a, *lda, s, u, *ldu, vt, *ldvt);
}

/* Cholesky factorisation A=L*L' (uplo 'L') or A=U'*U (uplo 'U'), in place. */
void dpotrf_(const char* uplo, ptrdiff_t* n, double* a, ptrdiff_t* lda, ptrdiff_t* info){
	const ptrdiff_t N=*n, ld=*lda;
	const int lower=(*uplo=='L'||*uplo=='l');
	*info=0;
	for(ptrdiff_t j=0; j<N; j++){
		double d=a[j+j*ld];
		for(ptrdiff_t k=0; k<j; k++){
			double l=lower?a[j+k*ld]:a[k+j*ld];
			d-=l*l;
		}
		if(d<=0){ *info=j+1; return; }
		d=sqrt(d);
		a[j+j*ld]=d;
		for(ptrdiff_t i=j+1; i<N; i++){
			double s=lower?a[i+j*ld]:a[j+i*ld];
			for(ptrdiff_t k=0; k<j; k++){
				s-=lower?a[i+k*ld]*a[j+k*ld]:a[k+i*ld]*a[k+j*ld];
			}
			if(lower) a[i+j*ld]=s/d; else a[j+i*ld]=s/d;
		}
	}
}
/* Solve A*X=B for symmetric positive definite A via dpotrf_. */
void dposv_(const char* uplo, const ptrdiff_t* n, const ptrdiff_t* nrhs, double* a, const ptrdiff_t* lda,
	double* b, const ptrdiff_t* ldb, ptrdiff_t* info){
	ptrdiff_t N=*n, ld=*lda;
	dpotrf_(uplo, &N, a, &ld, info);
	if(*info) return;
	const int lower=(*uplo=='L'||*uplo=='l');
	for(ptrdiff_t r=0; r<*nrhs; r++){
		double* x=b+r*(*ldb);
		for(ptrdiff_t i=0; i<N; i++){/* L y = b */
			double s=x[i];
			for(ptrdiff_t k=0; k<i; k++) s-=(lower?a[i+k*ld]:a[k+i*ld])*x[k];
			x[i]=s/a[i+i*ld];
		}
		for(ptrdiff_t i=N-1; i>=0; i--){/* L' x = y */
			double s=x[i];
			for(ptrdiff_t k=i+1; k<N; k++) s-=(lower?a[k+i*ld]:a[i+k*ld])*x[k];
			x[i]=s/a[i+i*ld];
		}
	}
}
/* Solve A*X=B by LU with partial pivoting (ipiv is 1-based as in LAPACK). */
void dgesv_(ptrdiff_t* n, ptrdiff_t* nrhs, double* a, ptrdiff_t* lda, ptrdiff_t* ipiv,
	double* b, ptrdiff_t* ldb, ptrdiff_t* info){
	const ptrdiff_t N=*n, ld=*lda;
	*info=0;
	for(ptrdiff_t j=0; j<N; j++){
		ptrdiff_t p=j;
		for(ptrdiff_t i=j+1; i<N; i++) if(fabs(a[i+j*ld])>fabs(a[p+j*ld])) p=i;
		ipiv[j]=p+1;
		if(a[p+j*ld]==0){ *info=j+1; return; }
		if(p!=j){
			for(ptrdiff_t k=0; k<N; k++){ double t=a[j+k*ld]; a[j+k*ld]=a[p+k*ld]; a[p+k*ld]=t; }
			for(ptrdiff_t r=0; r<*nrhs; r++){ double t=b[j+r*(*ldb)]; b[j+r*(*ldb)]=b[p+r*(*ldb)]; b[p+r*(*ldb)]=t; }
		}
		for(ptrdiff_t i=j+1; i<N; i++){
			double f=a[i+j*ld]/a[j+j*ld];
			a[i+j*ld]=f;
			for(ptrdiff_t k=j+1; k<N; k++) a[i+k*ld]-=f*a[j+k*ld];
			for(ptrdiff_t r=0; r<*nrhs; r++) b[i+r*(*ldb)]-=f*b[j+r*(*ldb)];
		}
	}
	for(ptrdiff_t r=0; r<*nrhs; r++){
		double* x=b+r*(*ldb);
		for(ptrdiff_t i=N-1; i>=0; i--){
			double s=x[i];
			for(ptrdiff_t k=i+1; k<N; k++) s-=a[i+k*ld]*x[k];
			x[i]=s/a[i+i*ld];
		}
	}
}

#define ABORT_STUB(name) void name(void){ fprintf(stderr, "oracle: reference called %s, which this build does not provide\n", #name); abort(); }
ABORT_STUB(sgemm_) ABORT_STUB(cgemm_)
ABORT_STUB(sgesvd_) ABORT_STUB(cgesvd_) ABORT_STUB(zgesvd_)
ABORT_STUB(sgesdd_) ABORT_STUB(cgesdd_) ABORT_STUB(zgesdd_)
ABORT_STUB(sgesv_) ABORT_STUB(cgesv_) ABORT_STUB(zgesv_)
ABORT_STUB(sposv_) ABORT_STUB(cposv_) ABORT_STUB(zposv_)
ABORT_STUB(spotrf_) ABORT_STUB(cpotrf_) ABORT_STUB(zpotrf_)
ABORT_STUB(chol_factorize) ABORT_STUB(chol_free_do) ABORT_STUB(chol_read)
ABORT_STUB(chol_save) ABORT_STUB(chol_solve) ABORT_STUB(chol_spsolve)
ABORT_STUB(zfft2) ABORT_STUB(zfft_free_plan) ABORT_STUB(sfft_free_plan)
const char* GIT_VERSION="oracle";
