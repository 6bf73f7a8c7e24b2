/*
 * Stand-in for the FFTW3 double-precision API, used only to compile the
 * reference's own math/fft.c into the test oracle (oracle/_ref).  FFTW itself
 * is a third-party dependency that the reference does not vendor and does not
 * pin (it installs libfftw3-dev from the distribution); it is absent here.
 *
 * Only the subset of the API that the reference's math/fft.c calls is
 * declared.  Conventions follow FFTW's published definition: FFTW_FORWARD is
 * exp(-2*pi*i*j*k/n), FFTW_BACKWARD is exp(+2*pi*i*j*k/n), no normalisation,
 * multi-dimensional plans are row-major (last dimension contiguous).
 *
 * This header is test infrastructure: nothing in the product includes it.
 */
#ifndef ORACLE_FFTW3_STANDIN_H
#define ORACLE_FFTW3_STANDIN_H
#include <stdio.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;
typedef struct fftw_iodim_do_not_use_me {
	int n;
	int is;
	int os;
} fftw_iodim;
typedef enum fftw_r2r_kind_do_not_use_me {
	FFTW_R2HC=0, FFTW_HC2R=1
} fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
	fftw_complex* in, const int* inembed, int istride, int idist,
	fftw_complex* out, const int* onembed, int ostride, int odist,
	int sign, unsigned flags);
fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim* dims,
	int howmany_rank, const fftw_iodim* howmany_dims,
	double* ri, double* ii, double* ro, double* io, unsigned flags);
fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_import_wisdom_from_file(FILE* f);
void fftw_export_wisdom_to_file(FILE* f);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
