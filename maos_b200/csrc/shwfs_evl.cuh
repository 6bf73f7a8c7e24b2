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
// (blocks, nevl), 256 threads; sums zeroed before the launch.
__global__ void __launch_bounds__(256) evl_sums_kernel(EvlRaster R, const float* __restrict__ opd, double* sums) {
	const int e = blockIdx.y;
	const long n = (long)R.nslot * 256;
	const float* o = opd + (size_t)e * n;
	double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
		const float a = R.amp[i];
		if (a == 0.f) continue;
		const int slot = (int)(i >> 8), p = (int)(i & 255);
		const int tile = R.slot_tile[slot];
		const int X = (tile % R.ntx) * 16 + (p & 15), Y = (tile / R.ntx) * 16 + (p >> 4);
		const double v = o[i], av = (double)a * v;
		s0 += av * v;
		s1 += av;
		s2 += av * (R.ox + X * R.dx);
		s3 += av * (R.oy + Y * R.dx);
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

// Radix-2 decimation-in-time FFT, forward (exp(-i), FFTW sign -1,
// unnormalised), of `rows` sequences of N points held in shared memory in
// bit-reversed order; output in natural order.  tw[k] = exp(-2 pi i k / N),
// k < N/2.
template <int N>
__device__ __forceinline__ void evl_fft_smem(float2* buf, int rows, const float2* __restrict__ tw) {
	const int nb = rows * (N / 2);
	for (int half = 1; half < N; half <<= 1) {
		const int tstride = N / (2 * half);
		for (int b = threadIdx.x; b < nb; b += blockDim.x) {
			const int r = b / (N / 2), q = b - r * (N / 2);
			const int grp = q / half, pos = q - grp * half;
			const int i = r * N + grp * 2 * half + pos, j = i + half;
			const float2 w = __ldg(tw + pos * tstride);
			const float2 u = buf[i], v = buf[j];
			const float2 t = make_float2(w.x * v.x - w.y * v.y, w.x * v.y + w.y * v.x);
			buf[i] = make_float2(u.x + t.x, u.y + t.y);
			buf[j] = make_float2(u.x - t.x, u.y - t.y);
		}
		__syncthreads();
	}
}

template <int N>
__device__ __forceinline__ int evl_brev(int i) {
	return (int)(__brev((unsigned)i) >> (33 - __ffs(N)));
}

// (3) PSF, first dimension (locfft_psf, lib/locfft.c:150-159): R raster
// rows per block, each embedded at column X + offx of an N-point row as
// amp * exp(i k (OPD - PTT)), transformed along x; the 2h columns the crop
// keeps are written to T (per direction, crop column ax major, row Y
// fastest).  Crop column ax takes frequency kx = ax < h ? N - h + ax : ax - h
// (the corner-to-centre copy).  Grid (ceil(nY / R), nevl).
template <int N, int R>
__global__ void __launch_bounds__(512) evl_psf_rows_kernel(EvlRaster Ra, const float* __restrict__ opd,
	const double* __restrict__ coeff, int pttr, float kwvl, int offx, int h, const float2* __restrict__ tw,
	float2* __restrict__ T, int nYp) {
	extern __shared__ float2 s_row[];
	const int e = blockIdx.y, Y0 = blockIdx.x * R;
	const float* o = opd + (size_t)e * Ra.nslot * 256;
	for (int i = threadIdx.x; i < R * N; i += blockDim.x) s_row[i] = make_float2(0.f, 0.f);
	__syncthreads();
	double c0 = 0, c1 = 0, c2 = 0;
	if (pttr) {
		c0 = coeff[e * 3];
		c1 = coeff[e * 3 + 1];
		c2 = coeff[e * 3 + 2];
	}
	for (int idx = threadIdx.x; idx < R * Ra.nX; idx += blockDim.x) {
		const int r = idx / Ra.nX, X = idx - r * Ra.nX, Y = Y0 + r;
		if (Y >= Ra.nY) continue;
		const int slot = Ra.tile_slot[(Y >> 4) * Ra.ntx + (X >> 4)];
		if (slot < 0) continue;
		const int p = slot * 256 + (Y & 15) * 16 + (X & 15);
		const float a = Ra.amp[p];
		if (a == 0.f) continue;
		float v = o[p];
		if (pttr) v = (float)((double)v - (c0 + c1 * (Ra.ox + X * Ra.dx) + c2 * (Ra.oy + Y * Ra.dx)));
		float sn, cs;
		sincosf(kwvl * v, &sn, &cs);
		s_row[r * N + evl_brev<N>(X + offx)] = make_float2(a * cs, a * sn);
	}
	__syncthreads();
	evl_fft_smem<N>(s_row, R, tw);
	const int ncol = 2 * h;
	float2* Te = T + (size_t)e * ncol * nYp;
	for (int idx = threadIdx.x; idx < R * ncol; idx += blockDim.x) {
		const int ax = idx / R, r = idx - ax * R, Y = Y0 + r;
		if (Y >= Ra.nY) continue;
		const int kx = ax < h ? N - h + ax : ax - h;
		Te[(size_t)ax * nYp + Y] = s_row[r * N + kx];
	}
}

// (4) PSF, second dimension: one block per kept column ax and direction;
// rows Y of T placed at Y + offy of an N-point column (zero elsewhere),
// transformed along y, |.|^2 of the 2h kept frequencies added to the sum
// psf (per direction, ax major, ay fastest).
template <int N>
__global__ void __launch_bounds__(512) evl_psf_cols_kernel(const float2* __restrict__ T, int nY, int nYp, int offy,
	int h, const float2* __restrict__ tw, float* __restrict__ psf) {
	extern __shared__ float2 s_col[];
	const int ax = blockIdx.x, e = blockIdx.y, ncol = 2 * h;
	const float2* Tc = T + ((size_t)e * ncol + ax) * nYp;
	for (int i = threadIdx.x; i < N; i += blockDim.x) s_col[i] = make_float2(0.f, 0.f);
	__syncthreads();
	for (int Y = threadIdx.x; Y < nY; Y += blockDim.x) s_col[evl_brev<N>(Y + offy)] = Tc[Y];
	__syncthreads();
	evl_fft_smem<N>(s_col, 1, tw);
	float* P = psf + ((size_t)e * ncol + ax) * ncol;
	for (int ay = threadIdx.x; ay < ncol; ay += blockDim.x) {
		const int ky = ay < h ? N - h + ay : ay - h;
		const float2 v = s_col[ky];
		P[ay] += v.x * v.x + v.y * v.y;
	}
}

// (5) OPD of one direction in aperture order.
__global__ void evl_gather_kernel(const float* __restrict__ opd, const int* __restrict__ loc_addr, long nloc,
	float* __restrict__ out) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < nloc) out[i] = opd[loc_addr[i]];
}

}  // namespace shwfs
