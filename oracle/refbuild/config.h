/* Minimal config.h for compiling the reference's C sources as a test oracle.
   Values describe this build: double precision, no CUDA, no FFTW threads,
   no zstd, no scheduler, no websockets. */
#ifndef ORACLE_REF_CONFIG_H
#define ORACLE_REF_CONFIG_H
#define CPU_SINGLE 0
#define USE_CPP 0
#define USE_CUDA 0
#define CUDA_DOUBLE 0
#define HAS_FFTWF 0
#define HAS_FFTW_THREADS 0
#define HAS_FFTW_CALLBACK 0
#define BIGENDIAN 0
#define MAOS_DISABLE_SCHEDULER 1
#define HAS_LWS 0
#define HAS_CMOCKA 0
#define MAC_INTEGRATION 0
#define COMPILER "gcc"
#define LDSUFFIX "so"
/* SRCDIR (the reference tree) comes from the oracle Makefile's REF */
#ifndef SRCDIR
#define SRCDIR "."
#endif
#define BUILDDIR "/tmp"
#define DEBUG 0
#define PACKAGE_VERSION "oracle"
#define PACKAGE "maos"
#endif
