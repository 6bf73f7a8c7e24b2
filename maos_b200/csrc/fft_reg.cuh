// Register-resident FFT building blocks for one thread.
//
// A thread holds a whole length-N sequence in registers and transforms it
// with a fully unrolled radix-2 Cooley-Tukey FFT.  Twiddles are compile-time
// constants (computed by constexpr Taylor series in double and rounded to
// float), so they become instruction immediates: no table loads, no shared
// memory, no shuffles.  Sign convention is FFTW's: DIR=-1 forward
// exp(-2*pi*i*j*k/N), DIR=+1 backward, no scaling.
#pragma once
#include <cuda_runtime.h>

namespace shwfs {

// ---- compile-time trigonometry (own Taylor-series evaluation) ----
constexpr double kPi = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double ct_sin_small(double x) {
	// x in [-pi/4, pi/4]; 14 terms reach double precision
	double term = x, sum = x, x2 = x * x;
	for (int n = 1; n < 14; n++) {
		term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
		sum += term;
	}
	return sum;
}
__host__ __device__ constexpr double ct_cos_small(double x) {
	double term = 1.0, sum = 1.0, x2 = x * x;
	for (int n = 1; n < 14; n++) {
		term *= -x2 / ((2.0 * n - 1.0) * (2.0 * n));
		sum += term;
	}
	return sum;
}
// cos(2*pi*k/n) and sin(2*pi*k/n) for integers, reduced to an octant so the
// series converges fast and symmetric values come out exactly symmetric.
__host__ __device__ constexpr double ct_cos2pi(long k, long n) {
	k %= n;
	if (k < 0) k += n;
	// use 8*k vs n to find the octant
	const long k8 = 8 * k;
	if (k8 <= n) return ct_cos_small(2.0 * kPi * (double)k / (double)n);
	if (k8 <= 3 * n) return -ct_sin_small(2.0 * kPi * (double)k / (double)n - kPi / 2);
	if (k8 <= 5 * n) return -ct_cos_small(2.0 * kPi * (double)k / (double)n - kPi);
	if (k8 <= 7 * n) return ct_sin_small(2.0 * kPi * (double)k / (double)n - 3 * kPi / 2);
	return ct_cos_small(2.0 * kPi * (double)k / (double)n - 2 * kPi);
}
// e^{DIR*2*pi*i*k/N} as float (requires N % 4 == 0 for the sine identity)
template <int DIR, int N, int K>
struct Tw {
	static constexpr float re = (float)ct_cos2pi(K, N);
	// sin(2 pi k/N) = cos(2 pi (k - N/4)/N)
	static constexpr float im = (float)(DIR * ct_cos2pi((long)K - N / 4, N));
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
	return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
	return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}

// multiply by the compile-time twiddle e^{DIR*2*pi*i*K/N}
template <int DIR, int N, int K>
__device__ __forceinline__ float2 twmul(float2 v) {
	constexpr int k = ((K % N) + N) % N;
	if constexpr (k == 0) {
		return v;
	} else if constexpr (4 * k == N) {  // DIR*i
		return DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
	} else if constexpr (2 * k == N) {  // -1
		return make_float2(-v.x, -v.y);
	} else if constexpr (4 * k == 3 * N) {  // -DIR*i
		return DIR < 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
	} else {
		constexpr float c = Tw<DIR, N, k>::re;
		constexpr float s = Tw<DIR, N, k>::im;
		return make_float2(fmaf(v.x, c, -v.y * s), fmaf(v.x, s, v.y * c));
	}
}

template <int N>
__host__ __device__ constexpr int ct_log2() {
	int l = 0;
	for (int n = N; n > 1; n >>= 1) l++;
	return l;
}
template <int BITS>
__host__ __device__ constexpr int ct_brev(int i) {
	int r = 0;
	for (int b = 0; b < BITS; b++) r |= ((i >> b) & 1) << (BITS - 1 - b);
	return r;
}

// One radix-2 stage of length LEN over the whole array (indices compile-time).
template <int DIR, int N, int LEN, int K>
__device__ __forceinline__ void fft_stage_k(float2 (&a)[N]) {
	if constexpr (K < LEN / 2) {
#pragma unroll
		for (int s = 0; s < N; s += LEN) {
			float2 u = a[s + K];
			float2 v = twmul<DIR, LEN, K>(a[s + K + LEN / 2]);
			a[s + K] = cadd(u, v);
			a[s + K + LEN / 2] = csub(u, v);
		}
		fft_stage_k<DIR, N, LEN, K + 1>(a);
	}
}
template <int DIR, int N, int LEN>
__device__ __forceinline__ void fft_stages(float2 (&a)[N]) {
	if constexpr (LEN <= N) {
		fft_stage_k<DIR, N, LEN, 0>(a);
		fft_stages<DIR, N, LEN * 2>(a);
	}
}
template <int N, int I>
__device__ __forceinline__ void bitrev_perm(float2 (&a)[N]) {
	if constexpr (I < N) {
		constexpr int J = ct_brev<ct_log2<N>()>(I);
		if constexpr (I < J) {
			float2 t = a[I];
			a[I] = a[J];
			a[J] = t;
		}
		bitrev_perm<N, I + 1>(a);
	}
}

// In-place length-N FFT of a register array (natural order in and out).
template <int DIR, int N>
__device__ __forceinline__ void fft_reg(float2 (&a)[N]) {
	bitrev_perm<N, 0>(a);
	fft_stages<DIR, N, 2>(a);
}

// Multiply element j of a length-N array by e^{DIR*2*pi*i*j*M/NN} (compile-time).
template <int DIR, int N, int NN, int M, int J>
__device__ __forceinline__ void twiddle_ramp_j(float2 (&a)[N]) {
	if constexpr (J < N) {
		a[J] = twmul<DIR, NN, J * M>(a[J]);
		twiddle_ramp_j<DIR, N, NN, M, J + 1>(a);
	}
}
template <int DIR, int N, int NN, int M>
__device__ __forceinline__ void twiddle_ramp(float2 (&a)[N]) {
	twiddle_ramp_j<DIR, N, NN, M, 0>(a);
}

}  // namespace shwfs
