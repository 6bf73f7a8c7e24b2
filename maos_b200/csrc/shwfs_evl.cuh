// Science-path kernels: wavefront-error sums and the PSF of the science
// aperture (open-loop performance evaluation, cuda/sim/perfevl.cu:336-509,
// maos/perfevl.c:111-240).
//
// The aperture (a regular grid) is held as 16x16 tiles: the tiles that hold
// aperture points get a slot, and the OPD of a direction is slot-major,
// 256 points per slot, row-major inside a tile.  geom_kernel traces the
// tiles like subapertures; points of a tile outside the aperture carry zero
// amplitude, so every sum below equals the one over the aperture points.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "shwfs_gen.cuh"

namespace shwfs {

struct EvlRaster {
	int nslot, ntx, nty, nX, nY;
	double ox, oy, dx;       // position of raster point (0, 0); spacing
	const int* tile_slot;    // ntx*nty: slot of a tile, or -1
	const int* slot_tile;    // nslot: tile of a slot (ty*ntx + tx)
	const float* amp;        // nslot*256
};

// (1) loc_calc_ptt_stride (math/loc.c:653-704) sums over the aperture, per
// direction: s = {sum a o^2, sum a o, sum a o x, sum a o y}, FP64; grid
// (ceil(nslot / EVL_SUM_TILES), nevl), 256 threads (one point of a tile
// each), EVL_SUM_TILES tiles per block with all their loads in flight; sums
// zeroed before the launch.
constexpr int EVL_SUM_TILES = 8;
__global__ void __launch_bounds__(256) evl_sums_kernel(EvlRaster R, const float* __restrict__ opd, double* sums) {
	const int e = blockIdx.y, p = threadIdx.x;
	const float* o = opd + (size_t)e * R.nslot * 256;
	const int slot0 = blockIdx.x * EVL_SUM_TILES;
	float av[EVL_SUM_TILES], ov[EVL_SUM_TILES];
#pragma unroll
	for (int k = 0; k < EVL_SUM_TILES; k++) {
		const int slot = slot0 + k;
		const size_t i = (size_t)slot * 256 + p;
		av[k] = slot < R.nslot ? __ldg(R.amp + i) : 0.f;
		ov[k] = slot < R.nslot ? __ldg(o + i) : 0.f;
	}
	double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
	for (int k = 0; k < EVL_SUM_TILES; k++) {
		if (av[k] == 0.f) continue;
		const int tile = R.slot_tile[slot0 + k];
		const int X = (tile % R.ntx) * 16 + (p & 15), Y = (tile / R.ntx) * 16 + (p >> 4);
		const double v = ov[k], a = (double)av[k] * v;
		s0 += a * v;
		s1 += a;
		s2 += a * (R.ox + X * R.dx);
		s3 += a * (R.oy + Y * R.dx);
	}
	__shared__ double red[4][8];
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) {
		s0 += __shfl_xor_sync(0xffffffffu, s0, off);
		s1 += __shfl_xor_sync(0xffffffffu, s1, off);
		s2 += __shfl_xor_sync(0xffffffffu, s2, off);
		s3 += __shfl_xor_sync(0xffffffffu, s3, off);
	}
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (lane == 0) {
		red[0][w] = s0;
		red[1][w] = s1;
		red[2][w] = s2;
		red[3][w] = s3;
	}
	__syncthreads();
	if (threadIdx.x < 4) {
		double t = 0;
		for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[threadIdx.x][k];
		atomicAdd(sums + e * 4 + threadIdx.x, t);
	}
}

// (2) mode coefficients for the PSF: coeff = imcc (s1, s2, s3)
// (dmulvec3 in loc_calc_ptt_stride); one thread per direction.
__global__ void evl_coeff_kernel(const double* __restrict__ sums, const double* __restrict__ imcc, double* coeff,
	int nevl) {
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= nevl) return;
	const double c[3] = {sums[e * 4 + 1], sums[e * 4 + 2], sums[e * 4 + 3]};
	for (int i = 0; i < 3; i++) coeff[e * 3 + i] = imcc[i] * c[0] + imcc[3 + i] * c[1] + imcc[6 + i] * c[2];
}

// Shared-memory rows of N points hold one pad element after every 16
// (evl_pad), so that the strided stores of the first Stockham passes fall on
// distinct banks.
template <int N>
__host__ __device__ constexpr int evl_row_len() { return N + N / 16; }
__device__ __forceinline__ int evl_pad(int i) { return i + (i >> 4); }

// Forward FFT (exp(-i), FFTW sign -1, unnormalised) of ROWS sequences of N
// points in shared memory, natural order in and out, by a block of
// EVL_THREADS threads: Stockham passes of radix 8 (and one of radix 2 or 4
// when log2 N is not a multiple of 3).  A radix-R pass reads the R points
// j + k N/R of group j into registers, applies the twiddles w^((j mod Ns) k)
// of the Ns*R-point stage and an R-point DFT, and writes them to
// (j / Ns) Ns R + (j mod Ns) + k Ns.  Each thread holds all its groups of a
// pass, so one barrier between the loads and the stores makes the pass in
// place.  tw[m] = exp(-2 pi i m / N), m < N.
constexpr int EVL_THREADS = 512;

template <int R>
__device__ __forceinline__ void evl_dft_small(float2 (&v)[R]) {
	if constexpr (R == 8) {
		dft8(v, -1.f);
	} else if constexpr (R == 4) {
		const float2 s0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y), d0 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
		const float2 s1 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y), d1 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
		const float2 d1r = make_float2(d1.y, -d1.x);  // d1 * (-i)
		v[0] = make_float2(s0.x + s1.x, s0.y + s1.y);
		v[1] = make_float2(d0.x + d1r.x, d0.y + d1r.y);
		v[2] = make_float2(s0.x - s1.x, s0.y - s1.y);
		v[3] = make_float2(d0.x - d1r.x, d0.y - d1r.y);
	} else {
		static_assert(R == 2, "radix 2, 4 or 8");
		const float2 a = v[0], b = v[1];
		v[0] = make_float2(a.x + b.x, a.y + b.y);
		v[1] = make_float2(a.x - b.x, a.y - b.y);
	}
}

// FIRST: the pass reads only row elements in [lo, hi) and takes the others
// as zero, so the rows need no zero fill.  LAST: the pass hands each output
// (row, index, value) to epi instead of storing it, so a crop reads no
// shared memory afterwards.
template <int N, int R, int ROWS, int Ns, bool FIRST, bool LAST, class Epi>
__device__ __forceinline__ void evl_stockham_pass(float2* buf, const float2* __restrict__ tw, int lo, int hi, Epi& epi) {
	constexpr int NG = N / R;  // groups per row
	constexpr int NGT = ROWS * NG;
	constexpr int GPT = (NGT + EVL_THREADS - 1) / EVL_THREADS;
	float2 v[GPT][R];
#pragma unroll
	for (int g = 0; g < GPT; g++) {
		const int gi = threadIdx.x + g * EVL_THREADS;
		if (gi < NGT) {
			const int row = gi / NG, j = gi - row * NG;
			const float2* x = buf + row * evl_row_len<N>();
			const int jm = j % Ns, tstep = jm * (N / (Ns * R));
#pragma unroll
			for (int k = 0; k < R; k++) {
				const int xi = j + k * NG;
				if (FIRST)
					v[g][k] = (xi >= lo && xi < hi) ? x[evl_pad(xi)] : make_float2(0.f, 0.f);
				else
					v[g][k] = x[evl_pad(xi)];
			}
			if (jm) {
				// w^k for k < R from w, w^2 and w^4 of the table (two roundings at most)
				float2 w[R];
				w[1] = __ldg(tw + tstep);
				if constexpr (R >= 4) {
					w[2] = __ldg(tw + 2 * tstep);
					w[3] = cmul(w[1], w[2]);
				}
				if constexpr (R == 8) {
					w[4] = __ldg(tw + 4 * tstep);
					w[5] = cmul(w[1], w[4]);
					w[6] = cmul(w[2], w[4]);
					w[7] = cmul(w[3], w[4]);
				}
#pragma unroll
				for (int k = 1; k < R; k++) v[g][k] = cmul(v[g][k], w[k]);
			}
			evl_dft_small<R>(v[g]);
		}
	}
	if constexpr (LAST) {
#pragma unroll
		for (int g = 0; g < GPT; g++) {
			const int gi = threadIdx.x + g * EVL_THREADS;
			if (gi < NGT) {
				const int row = gi / NG, j = gi - row * NG;
				const int jm = j % Ns, base = (j / Ns) * Ns * R + jm;
#pragma unroll
				for (int k = 0; k < R; k++) epi(row, base + k * Ns, v[g][k]);
			}
		}
	} else {
		__syncthreads();
#pragma unroll
		for (int g = 0; g < GPT; g++) {
			const int gi = threadIdx.x + g * EVL_THREADS;
			if (gi < NGT) {
				const int row = gi / NG, j = gi - row * NG;
				float2* y = buf + row * evl_row_len<N>();
				const int jm = j % Ns, base = (j / Ns) * Ns * R + jm;
#pragma unroll
				for (int k = 0; k < R; k++) y[evl_pad(base + k * Ns)] = v[g][k];
			}
		}
		__syncthreads();
	}
}

template <int N>
__host__ __device__ constexpr int evl_log2() {
	return (N >= 4096) ? 12 : (N >= 2048) ? 11 : (N >= 1024) ? 10 : (N >= 512) ? 9 : (N >= 256) ? 8 : (N >= 128) ? 7 : 6;
}

// Pass P of the transform and the passes after it: log2(N)/3 radix-8
// passes, then one radix-4 or radix-2 pass when log2 N is not a multiple of 3.
template <int N, int ROWS, int P, int Ns, class Epi>
__device__ __forceinline__ void evl_fft_passes(float2* buf, const float2* __restrict__ tw, int lo, int hi, Epi& epi) {
	constexpr int L = evl_log2<N>();
	constexpr int NP8 = L / 3;
	constexpr int NPASS = NP8 + (L % 3 ? 1 : 0);
	constexpr int RP = P < NP8 ? 8 : (L % 3 == 2 ? 4 : 2);
	evl_stockham_pass<N, RP, ROWS, Ns, P == 0, P == NPASS - 1>(buf, tw, lo, hi, epi);
	if constexpr (P + 1 < NPASS) evl_fft_passes<N, ROWS, P + 1, Ns * RP>(buf, tw, lo, hi, epi);
}

// Forward transform of ROWS rows whose elements outside [lo, hi) are zero
// (not read); output (row, k, X[k]) goes to epi.
template <int N, int ROWS, class Epi>
__device__ __forceinline__ void evl_fft_smem(float2* buf, const float2* __restrict__ tw, int lo, int hi, Epi& epi) {
	static_assert((1 << evl_log2<N>()) == N, "N must be a power of two in [64, 4096]");
	evl_fft_passes<N, ROWS, 0, 1>(buf, tw, lo, hi, epi);
}

// Column of the corner-to-centre crop that frequency k lands in (the crop
// keeps kx = ax < h ? N - h + ax : ax - h), or -1.
template <int N>
__device__ __forceinline__ int evl_crop_index(int k, int h) {
	return k < h ? k + h : (k >= N - h ? k - (N - h) : -1);
}

// (3) PSF, first dimension (locfft_psf, lib/locfft.c:150-159): R raster
// rows per block (512 threads), each embedded at column X + offx of an N-point row as
// amp * exp(i 2 pi (OPD - PTT) / wvl), transformed along x; the 2h columns the crop
// keeps are written to T (per direction, crop column ax major, row Y
// fastest) straight from the last pass.  Grid (ceil(nY / R), nevl).
template <int N, int R>
__global__ void __launch_bounds__(EVL_THREADS, 4) evl_psf_rows_kernel(EvlRaster Ra, const float* __restrict__ opd,
	const double* __restrict__ coeff, int pttr, float twoinvwvl, int offx, int h, const float2* __restrict__ tw,
	float2* __restrict__ T, int nYp) {
	extern __shared__ float2 s_row[];
	const int e = blockIdx.y, Y0 = blockIdx.x * R;
	const float* o = opd + (size_t)e * Ra.nslot * 256;
	constexpr int LN = evl_row_len<N>();
	double c0 = 0, c1 = 0, c2 = 0;
	if (pttr) {
		c0 = coeff[e * 3];
		c1 = coeff[e * 3 + 1];
		c2 = coeff[e * 3 + 2];
	}
	// the field on columns [offx, offx + nX) of every row (zero where the
	// aperture has no point); U elements of a row per thread in flight
	const int nX = Ra.nX;
	constexpr int U = 4;
#pragma unroll 1
	for (int r = 0; r < R; r++) {
		const int Y = Y0 + r;
		float2* srow = s_row + r * LN;
		if (Y >= Ra.nY) {
			for (int X = threadIdx.x; X < nX; X += EVL_THREADS) srow[evl_pad(X + offx)] = make_float2(0.f, 0.f);
			continue;
		}
		const int* trow = Ra.tile_slot + (Y >> 4) * Ra.ntx;
		const int py = (Y & 15) * 16;
		for (int X0 = threadIdx.x; X0 < nX; X0 += U * EVL_THREADS) {
			int pp[U];
#pragma unroll
			for (int u = 0; u < U; u++) {
				const int X = X0 + u * EVL_THREADS;
				pp[u] = -1;
				if (X < nX) {
					const int slot = trow[X >> 4];
					if (slot >= 0) pp[u] = slot * 256 + py + (X & 15);
				}
			}
			float av[U], ov[U];
#pragma unroll
			for (int u = 0; u < U; u++) {
				av[u] = pp[u] >= 0 ? Ra.amp[pp[u]] : 0.f;
				ov[u] = pp[u] >= 0 ? o[pp[u]] : 0.f;
			}
#pragma unroll
			for (int u = 0; u < U; u++) {
				const int X = X0 + u * EVL_THREADS;
				if (X < nX) {
					float2 val = make_float2(0.f, 0.f);
					if (av[u] != 0.f) {
						float v = ov[u];
						if (pttr) v = (float)((double)v - (c0 + c1 * (Ra.ox + X * Ra.dx) + c2 * (Ra.oy + Y * Ra.dx)));
						float sn, cs;
						sincospif(twoinvwvl * v, &sn, &cs);  // exp(i 2 pi v / wvl)
						val = make_float2(av[u] * cs, av[u] * sn);
					}
					srow[evl_pad(X + offx)] = val;
				}
			}
		}
	}
	__syncthreads();
	float2* Te = T + (size_t)e * (2 * h) * nYp;
	auto crop = [&](int r, int kx, float2 v) {
		const int ax = evl_crop_index<N>(kx, h), Y = Y0 + r;
		if (ax >= 0 && Y < Ra.nY) Te[(size_t)ax * nYp + Y] = v;
	};
	evl_fft_smem<N, R>(s_row, tw, offx, offx + nX, crop);
}

// (4) PSF, second dimension: one block per kept column ax and direction;
// rows Y of T placed at Y + offy of an N-point column (zero elsewhere),
// transformed along y, |.|^2 of the 2h kept frequencies added to the sum
// psf (per direction, ax major, ay fastest) straight from the last pass.
template <int N>
__global__ void __launch_bounds__(EVL_THREADS, 4) evl_psf_cols_kernel(const float2* __restrict__ T, int nY, int nYp, int offy,
	int h, const float2* __restrict__ tw, float* __restrict__ psf) {
	extern __shared__ float2 s_col[];
	const int ax = blockIdx.x, e = blockIdx.y, ncol = 2 * h;
	const float2* Tc = T + ((size_t)e * ncol + ax) * nYp;
#pragma unroll 4
	for (int Y = threadIdx.x; Y < nY; Y += EVL_THREADS) s_col[evl_pad(Y + offy)] = __ldg(Tc + Y);
	__syncthreads();
	float* P = psf + ((size_t)e * ncol + ax) * ncol;
	auto acc = [&](int, int ky, float2 v) {
		const int ay = evl_crop_index<N>(ky, h);
		if (ay >= 0) P[ay] += v.x * v.x + v.y * v.y;
	};
	evl_fft_smem<N, 1>(s_col, tw, offy, offy + nY, acc);
}

// (5) OPD of one direction in aperture order.
__global__ void evl_gather_kernel(const float* __restrict__ opd, const int* __restrict__ loc_addr, long nloc,
	float* __restrict__ out) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < nloc) out[i] = opd[loc_addr[i]];
}

}  // namespace shwfs
