// Matched-filter regeneration on the device, 32-point path (n_o = 16, n_f =
// 32): the reference builds i0 and its derivatives (lib/gensei.c:213-419) and
// the matched filter (lib/mtch.c:93-211 mtch, :223-335 mtch_cell) on the host
// and copies them in (gpu_wfsgrad_update_ref, cuda/sim/gpu_sim.h:42); here
// they are formed from the device-resident amplitude, transfer functions and
// short-exposure OTF, so a sodium-profile or reference update needs no host
// round trip.  The short-exposure OTF of each subaperture (turbulence with
// piston/tip/tilt removed times the conjugate uplink OTF, as genseotf and
// gensepsf form it, lib/gensei.c:41-209) is static and uploaded once
// (shwfs_powfs_set_seotf); without it the images are those of a flat
// wavefront.
//
//   mtch_images_kernel: one warp per subaperture; the short-exposure OTF (or
//     the OTF of the flat field x conj(flat uplink OTF)) x ETF / nominal,
//     times 1, Ux(fx), Ux(fy) with Ux(f) = -2 pi i f' / (dtheta n) (f' the
//     signed frequency), inverse FFT, real part, pixel map, x the signal
//     level (x norm_ints for the flat field) -> i0, gx, gy; i0 sums and max.
//   mtch_filter_kernel: one warp per subaperture; A = [gx, gy, i0 kp + 2 bkg,
//     (i0 shifted by +-1 pixel in x, y)], W = 1 / (rne^2 + bkg + i0), the
//     weighted pseudo-inverse (A'WA)^-1 A'W with the eigenvalue thresholds of
//     dpinv (math/blas.c:170-205: 1e-7 absolute, 1e-3 relative to the previous
//     kept one), mtche = the x and y rows, zeroed for dim subapertures (i0 sum
//     below max(0.1 max, 10 rne)) or noise-equivalent angles above 10 pixels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "shwfs_kernels.cuh"

namespace shwfs {

constexpr int MTCH_MAXMOD = 7;

struct MtchParams {
	int nsa, npix, pixpsax, pixpsay;
	int nmod, crx, cry;           // columns of A and the positions of the shifted-i0 pairs (0: none)
	float norm_ints, dux;         // sigsim norm_psf^2 / n^2, 1 / (dtheta n)
	const float* amp;             // nsa * 256
	const float* zero_opd;        // 256 zeros
	const float2* lotfT;          // flat uplink OTF (transposed), or null
	const float2* seotfT;         // nsa * 1024 short-exposure OTF (transposed), or null: flat wavefront
	const float2* etfT1;          // nsa * 1024 transposed, or null
	const float2* etfT2;
	float etfwt1, etfwt2;
	const float* nominalT;        // 1024 (or nsa * 1024) transposed, or null
	int nominal_per_sa;
	const int* simap_idx;         // npix * 4 (shared by the subapertures)
	const float* simap_wt;
	double kpx, kpy, bkgrnd, bkgrnd_res, rne, nea2thres;
	float* img;                   // nsa * 3 * npix scratch: i0, gx, gy
	float* i0sum;                 // nsa
	unsigned* i0max_bits;         // max of the positive i0 sums (float bits)
	double* i0sumsum;
	float* mtche;                 // nsa * 2 * npix, [isa][r + 2 p]
};

template <int NPQ>
__global__ void __launch_bounds__(128) mtch_images_kernel(MtchParams M) {
	__shared__ float2 tiles[4][32 * LD];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int isa = blockIdx.x * 4 + warp;
	if (isa >= M.nsa) return;
	float2* tile = tiles[warp];
	float2 F[32];
	if (M.seotfT) {  // the short-exposure OTF of turbulence and uplink (genseotf, gensepsf)
		const float2* so = M.seotfT + (size_t)isa * 1024 + lane;
#pragma unroll
		for (int fx = 0; fx < 32; fx++) F[fx] = __ldg(so + 32 * fx);
	} else {
		field_fft_n32(M.zero_opd, M.amp + (size_t)isa * 256, 0.f, tile, lane, F);
		psf_to_otf_n32(F, 1.f, tile, lane);  // lane = fy holds OTF(fx, fy) in F[fx]
		if (M.lotfT) {
#pragma unroll
			for (int fx = 0; fx < 32; fx++) F[fx] = cmulc(F[fx], __ldg(M.lotfT + lane + 32 * fx));
		}
	}
	if (M.etfT1) {
		const float2* e1 = M.etfT1 + (size_t)isa * 1024 + lane;
#pragma unroll
		for (int fx = 0; fx < 32; fx++) {
			float2 e = __ldg(e1 + 32 * fx);
			if (M.etfT2) {
				const float2 f = __ldg(M.etfT2 + (size_t)isa * 1024 + lane + 32 * fx);
				e = make_float2(e.x * M.etfwt1 + f.x * M.etfwt2, e.y * M.etfwt1 + f.y * M.etfwt2);
			}
			F[fx] = cmul(F[fx], e);
		}
	} else if (M.nominalT) {
		const float* nm = M.nominalT + (M.nominal_per_sa ? (size_t)isa * 1024 : 0) + lane;
#pragma unroll
		for (int fx = 0; fx < 32; fx++) {
			const float d = __ldg(nm + 32 * fx);
			F[fx] = make_float2(F[fx].x * d, F[fx].y * d);
		}
	}
	const float two_pi_dux = 6.283185307179586f * M.dux;
	const float uy = -two_pi_dux * (float)(lane < 16 ? lane : lane - 32);  // Ux(fy), fy = lane
#pragma unroll 1
	for (int d = 0; d < 3; d++) {
		float2 G[32];
#pragma unroll
		for (int fx = 0; fx < 32; fx++) {
			const float u = d == 1 ? -two_pi_dux * (float)(fx < 16 ? fx : fx - 32) : uy;
			G[fx] = d == 0 ? F[fx] : make_float2(-u * F[fx].y, u * F[fx].x);  // x (i u)
		}
		fft_reg<1, 32>(G);
		__syncwarp();
#pragma unroll
		for (int k = 0; k < 32; k++) tile[k * LD + lane] = G[k];  // tile[x][fy]
		__syncwarp();
#pragma unroll
		for (int k = 0; k < 32; k++) G[k] = tile[lane * LD + k];  // lane = x
		fft_reg<1, 32>(G);
		__syncwarp();
		float* psf = reinterpret_cast<float*>(tile);  // psf[x + 32 y], real part
#pragma unroll
		for (int y = 0; y < 32; y++) psf[lane + 32 * y] = G[y].x;
		__syncwarp();
		float s = 0.f;
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < M.npix) {
				float v = 0.f;
#pragma unroll
				for (int c = 0; c < 4; c++) {
					const int id = __ldg(M.simap_idx + 4 * p + c);
					if (id >= 0) v = fmaf(__ldg(M.simap_wt + 4 * p + c), psf[id], v);
				}
				v *= M.norm_ints;
				M.img[((size_t)isa * 3 + d) * M.npix + p] = v;
				s += v;
			}
		}
		__syncwarp();
		if (d == 0) {
#pragma unroll
			for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
			if (lane == 0) {
				M.i0sum[isa] = s;
				if (s > 0.f) atomicMax(M.i0max_bits, __float_as_uint(s));
				atomicAdd(M.i0sumsum, (double)s);
			}
		}
	}
}

// Eigen-decomposition of a symmetric n x n matrix (column-major, n <= 7) by
// cyclic Jacobi rotations, as the project's host setup: a is destroyed, w gets
// the eigenvalues, v the eigenvectors (columns).
__device__ inline void jacobi_sym(double* a, int n, double* w, double* v) {
	for (int i = 0; i < n * n; i++) v[i] = 0;
	for (int i = 0; i < n; i++) v[i + i * n] = 1;
	for (int sweep = 0; sweep < 100; sweep++) {
		double off = 0, diag = 0;
		for (int p = 0; p < n; p++) {
			diag += a[p + p * n] * a[p + p * n];
			for (int q = p + 1; q < n; q++) off += a[p + q * n] * a[p + q * n];
		}
		if (off <= 1e-30 * diag || off == 0) break;
		for (int p = 0; p < n - 1; p++)
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
	for (int i = 0; i < n; i++) w[i] = a[i + i * n];
}

// column k of A at pixel p (i0, gx, gy of the subaperture in s_i0 / gx / gy)
__device__ __forceinline__ double mtch_col(const MtchParams& M, const float* s_i0, float gx, float gy, int k, int p) {
	if (k == 0) return gx;
	if (k == 1) return gy;
	if (k == 2) return (double)s_i0[p] * M.kpx + 2 * M.bkgrnd_res;
	const int nx = M.pixpsax, ny = M.pixpsay, ix = p % nx, iy = p / nx;
	double v = M.bkgrnd_res;
	if (M.crx && (k == M.crx || k == M.crx + 1)) {  // mki0sh(i0, kpx, 1, 0), lib/mtch.c:23-34
		if (k == M.crx && ix >= 1) v += (double)s_i0[p - 1] * M.kpx;
		if (k == M.crx + 1 && ix + 1 < nx) v += (double)s_i0[p + 1] * M.kpx;
		return v;
	}
	if (k == M.cry && iy >= 1) v += (double)s_i0[p - nx] * M.kpy;
	if (k == M.cry + 1 && iy + 1 < ny) v += (double)s_i0[p + nx] * M.kpy;
	return v;
}

template <int NPQ>
__global__ void __launch_bounds__(128) mtch_filter_kernel(MtchParams M) {
	__shared__ float s_i0s[4][128];
	__shared__ double s_inv[4][MTCH_MAXMOD * MTCH_MAXMOD];
	__shared__ int s_reject[4];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int isa = blockIdx.x * 4 + warp;
	if (isa >= M.nsa) return;
	const int npix = M.npix, nmod = M.nmod;
	float* s_i0 = s_i0s[warp];
	const float* img = M.img + (size_t)isa * 3 * npix;
	float gx[NPQ], gy[NPQ];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		if (p < npix) {
			s_i0[p] = img[p];
			gx[q] = img[npix + p];
			gy[q] = img[2 * npix + p];
		}
	}
	__syncwarp();
	const double rne2 = M.rne * M.rne;
	// normal matrix A'WA (upper triangle), FP64
	double cc[MTCH_MAXMOD * (MTCH_MAXMOD + 1) / 2];
#pragma unroll
	for (int k = 0; k < MTCH_MAXMOD * (MTCH_MAXMOD + 1) / 2; k++) cc[k] = 0;
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		if (p < npix) {
			const double i0 = s_i0[p];
			const double wt = i0 < 0 ? 1. / rne2 : 1. / (rne2 + M.bkgrnd + i0);
			double a[MTCH_MAXMOD];
#pragma unroll
			for (int k = 0; k < MTCH_MAXMOD; k++) a[k] = k < nmod ? mtch_col(M, s_i0, gx[q], gy[q], k, p) : 0.;
			int idx = 0;
#pragma unroll
			for (int i = 0; i < MTCH_MAXMOD; i++)
#pragma unroll
				for (int j = i; j < MTCH_MAXMOD; j++) cc[idx++] += a[i] * wt * a[j];
		}
	}
#pragma unroll
	for (int k = 0; k < MTCH_MAXMOD * (MTCH_MAXMOD + 1) / 2; k++)
#pragma unroll
		for (int off = 16; off > 0; off >>= 1) cc[k] += __shfl_xor_sync(0xffffffffu, cc[k], off);
	if (lane == 0) {
		double A[MTCH_MAXMOD * MTCH_MAXMOD], ev[MTCH_MAXMOD * MTCH_MAXMOD], ew[MTCH_MAXMOD];
		int idx = 0;
		for (int i = 0; i < MTCH_MAXMOD; i++)
			for (int j = i; j < MTCH_MAXMOD; j++, idx++)
				if (i < nmod && j < nmod) A[i + j * nmod] = A[j + i * nmod] = cc[idx];
		jacobi_sym(A, nmod, ew, ev);
		int ord[MTCH_MAXMOD];
		for (int i = 0; i < nmod; i++) ord[i] = i;
		for (int i = 0; i < nmod; i++)
			for (int j = i + 1; j < nmod; j++)
				if (fabs(ew[ord[j]]) > fabs(ew[ord[i]])) {
					const int t = ord[i];
					ord[i] = ord[j];
					ord[j] = t;
				}
		const double maxeig = fabs(ew[ord[0]]);
		const double thres10 = 1e-7 * maxeig;
		double thres20 = 1e-3 * maxeig;
		double sinv[MTCH_MAXMOD];
		for (int k = 0; k < nmod; k++) sinv[k] = 0;
		for (int k = 0; k < nmod; k++) {
			const double sv = fabs(ew[ord[k]]);
			if (sv > thres10 && sv > thres20) {
				thres20 = sv * 1e-3;
				sinv[k] = 1. / ew[ord[k]];
			} else {
				break;
			}
		}
		for (int i = 0; i < nmod; i++)
			for (int j = 0; j < nmod; j++) {
				double v = 0;
				for (int k = 0; k < nmod; k++) v += ev[i + ord[k] * nmod] * sinv[k] * ev[j + ord[k] * nmod];
				s_inv[warp][i + j * nmod] = v;
			}
		const float i0max = __uint_as_float(*M.i0max_bits);
		const double i0thres = fmax((double)i0max * 0.1, 10 * M.rne);
		s_reject[warp] = (double)M.i0sum[isa] < i0thres;
	}
	__syncwarp();
	// mtche = rows x, y of (i0m P), P = inv A'W; then the noise-equivalent angles
	const double* inv = s_inv[warp];
	double m0[NPQ], m1[NPQ], nea0 = 0, nea1 = 0;
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		m0[q] = m1[q] = 0;
		if (p < npix) {
			const double i0 = s_i0[p];
			const double wt = i0 < 0 ? 1. / rne2 : 1. / (rne2 + M.bkgrnd + i0);
			double a[MTCH_MAXMOD];
#pragma unroll
			for (int k = 0; k < MTCH_MAXMOD; k++) a[k] = k < nmod ? mtch_col(M, s_i0, gx[q], gy[q], k, p) : 0.;
			for (int k = 0; k < nmod; k++) {
				double P = 0;
				for (int j = 0; j < nmod; j++) P += inv[k + j * nmod] * a[j];
				P *= wt;
				// i0m: (1,0) gx, (0,1) gy, (0,0) i0, (1,0)/(-1,0) x pair, (0,1)/(0,-1) y pair
				if (k == 0 || (M.crx && k == M.crx)) m0[q] += P;
				if (M.crx && k == M.crx + 1) m0[q] -= P;
				if (k == 1 || (M.cry && k == M.cry)) m1[q] += P;
				if (M.cry && k == M.cry + 1) m1[q] -= P;
			}
			nea0 += m0[q] * m0[q] / wt;
			nea1 += m1[q] * m1[q] / wt;
		}
	}
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) {
		nea0 += __shfl_xor_sync(0xffffffffu, nea0, off);
		nea1 += __shfl_xor_sync(0xffffffffu, nea1, off);
	}
	const bool reject = s_reject[warp] || nea0 > M.nea2thres || nea1 > M.nea2thres;
	float* out = M.mtche + (size_t)isa * 2 * npix;
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		if (p < npix) {
			out[2 * p] = reject ? 0.f : (float)m0[q];
			out[2 * p + 1] = reject ? 0.f : (float)m1[q];
		}
	}
}

}  // namespace shwfs
