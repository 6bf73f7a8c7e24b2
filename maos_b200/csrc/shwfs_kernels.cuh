// Device kernels of the Shack-Hartmann frame.
//
//   raytrace_kernel     (a) bilinear gather of every turbulence layer into the
//                           subaperture OPD points, FP64 offsets
//   uplink_otf_kernel   LGS uplink OTF from the LLT OPD (one warp per WFS)
//   ints_n32_kernel     (b)-(e) fused per subaperture for n_w = n_f = 32,
//                           n_opd = 16: field, pruned 2-D FFT, |.|^2, FFT,
//                           x conj(uplink OTF) x ETF/DTF, inverse FFT, pixel
//                           sampling, Philox noise, CoG / matched filter
//   grad_kernel         (e) alone, from given pixel intensities
//
// One warp owns one subaperture image in ints_n32_kernel.  Each lane keeps a
// full 32-point sequence in registers and transforms it with the unrolled FFT
// of fft_reg.cuh; the warp moves data between the row and column passes
// through a padded 32x33 shared-memory tile, so no pass needs shuffles.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fft_reg.cuh"

namespace shwfs {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter-based generator.
// ---------------------------------------------------------------------------
struct u32x4 {
	uint32_t x, y, z, w;
};
__device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
	const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
	const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
	for (int r = 0; r < 10; r++) {
		const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
		const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
		c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
		k0 += W0;
		k1 += W1;
	}
	return c;
}
// uniform in (0, 1]: never 0, so a running product of draws stays positive
__device__ __forceinline__ float u01(uint32_t v) { return ((v >> 8) + 1u) * (1.0f / 16777216.0f); }

// Stream of uniforms for one pixel: counter (n, pixel, wfs, frame).
struct PixelRng {
	uint32_t k0, k1, pix, wfs, frame, n;
	u32x4 buf;
	int used;
	__device__ __forceinline__ PixelRng(uint64_t seed, uint32_t pix_, uint32_t wfs_, uint32_t frame_)
		: k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), pix(pix_), wfs(wfs_), frame(frame_), n(0), used(4) {}
	__device__ __forceinline__ float next() {
		if (used == 4) {
			buf = philox4x32_10(u32x4{n++, pix, wfs, frame}, k0, k1);
			used = 0;
		}
		uint32_t v = used == 0 ? buf.x : used == 1 ? buf.y : used == 2 ? buf.z : buf.w;
		used++;
		return u01(v);
	}
	// standard normal by Box-Muller
	__device__ __forceinline__ float normal() {
		float u1 = next(), u2 = next();
		float r = sqrtf(-2.f * logf(u1));
		float s, c;
		sincospif(2.f * u2, &s, &c);
		return r * c;
	}
};

// Poisson draw with the reference's method (math/random.c:186-209): a
// Gaussian approximation above 200, otherwise products of uniforms in chunks
// of at most 12.  The inner loop is capped; a draw that reaches the cap
// returns the count so far (probability below 1e-30 for these means).
__device__ __forceinline__ float poisson_draw(PixelRng& rng, float xm) {
	if (xm > 200.f) {
		return rintf(xm + rng.normal() * sqrtf(xm));
	}
	int x = 0;
	int guard = 0;
	while (xm > 0.f && guard < 4096) {
		const float xmu = xm > 12.f ? 12.f : xm;
		xm -= xmu;
		const float g = expf(-xmu);
		int xu = -1;
		float t = 1.f;
		while (t > g && guard < 4096) {
			xu++;
			t *= rng.next();
			guard++;
		}
		x += xu;
	}
	return (float)x;
}

// ---------------------------------------------------------------------------
// Parameters
// ---------------------------------------------------------------------------
// Per-layer ray-trace geometry for one WFS at one frame, computed on the host
// in FP64 (lib/accphi.c:241-244 and lib/accphi_grid_do.c:424-434).
struct LayerGeom {
	const float* screen;
	int nx, ny;
	double dispx, dispy;  // (displacement - screen origin)/screen dx, in screen pixels
	double sx;            // scale/screen dx   (multiplies point coordinates)
	float alpha;
};
#define SHWFS_MAX_LAYERS 16

struct RaytraceParams {
	const double* origx;  // nsa
	const double* origy;
	double dx;            // pts->dx
	int nopd, nsa;
	int nlayer;
	LayerGeom layer[SHWFS_MAX_LAYERS];
	float* opd;           // nsa*nopd^2
};

struct WfsDev {
	const float* opd;      // nsa*nopd^2
	const float* amp;      // nsa*nopd^2
	const float2* lotfT;   // notf^2, transposed (fy fastest), or null
	const float* mtche;    // nsa*2*npix
	const float* i0sum;    // nsa
	float* ints;           // nsa*npix, or null
	float* grad;           // 2*nsa, or null
	float alpha;           // sigsim*wvlwt*norm_psf^2/notf^2
	int noisy;
	uint32_t wfs_id;
	uint64_t seed;
};

struct PowfsDev {
	int nsa, npix, pixpsax, pixpsay;
	const float2* etfT1;   // nsa*notf^2 transposed, or null
	const float2* etfT2;   // second ETF for interpolation, or null
	float etfwt1, etfwt2;
	const float* nominalT; // notf^2 transposed (or nsa*notf^2), or null
	int nominal_per_sa;
	const int* simap_idx;  // nmap*npix*4
	const float* simap_wt;
	int simap_per_sa;
	int gradtype, sigmatch;
	float cogthres, cogoff, pixthetax, pixthetay, saat, sigtot;
	const float* saa;
	float twoinvwvl;       // 2/wvl: phase/pi per metre of OPD
	float rne, bkgrnd, bkgrndc;
	int isim;
	float lltnorm;         // 1/nlwvf^2 for the uplink PSF
};

// ---------------------------------------------------------------------------
// (a) ray trace
// ---------------------------------------------------------------------------
// One thread per OPD point, looping over layers; block = one subaperture's
// nopd^2 points (blockDim.x = nopd*nopd <= 1024).  The per-subaperture start
// coordinate is formed and wrapped in FP64; only the in-subaperture offset
// (< nopd screen pixels) is carried in FP32.
__global__ void raytrace_kernel(RaytraceParams p) {
	const int isa = blockIdx.x;
	const int ip = threadIdx.x;
	if (isa >= p.nsa || ip >= p.nopd * p.nopd) return;
	const int ix = ip % p.nopd, iy = ip / p.nopd;
	const double ox = p.origx[isa], oy = p.origy[isa];
	float acc = 0.f;
	for (int l = 0; l < p.nlayer; l++) {
		const LayerGeom& g = p.layer[l];
		// start of this subaperture in screen pixels, wrapped into [0, n)
		double x0 = ox * g.sx + g.dispx;
		double y0 = oy * g.sx + g.dispy;
		if (!isfinite(x0) || !isfinite(y0)) continue;
		x0 -= floor(x0 / g.nx) * g.nx;
		y0 -= floor(y0 / g.ny) * g.ny;
		const int ix0 = (int)floor(x0), iy0 = (int)floor(y0);
		const float fx0 = (float)(x0 - ix0), fy0 = (float)(y0 - iy0);
		const float step = (float)(p.dx * g.sx);
		const float xf = fx0 + ix * step;
		const float yf = fy0 + iy * step;
		const float flx = floorf(xf), fly = floorf(yf);
		int jx = ix0 + (int)flx, jy = iy0 + (int)fly;
		const float wx = xf - flx, wy = yf - fly;
		while (jx >= g.nx) jx -= g.nx;
		while (jy >= g.ny) jy -= g.ny;
		while (jx < 0) jx += g.nx;
		while (jy < 0) jy += g.ny;
		const int jx1 = jx == g.nx - 1 ? 0 : jx + 1;
		const int jy1 = jy == g.ny - 1 ? 0 : jy + 1;
		const float* s = g.screen;
		const float m00 = __ldg(s + jx + (size_t)g.nx * jy);
		const float m10 = __ldg(s + jx1 + (size_t)g.nx * jy);
		const float m01 = __ldg(s + jx + (size_t)g.nx * jy1);
		const float m11 = __ldg(s + jx1 + (size_t)g.nx * jy1);
		acc += g.alpha * ((m00 + (m10 - m00) * wx) * (1.f - wy) + (m01 + (m11 - m01) * wx) * wy);
	}
	p.opd[(size_t)isa * p.nopd * p.nopd + ip] = acc;
}

// ---------------------------------------------------------------------------
// Shared pieces of the 32-point pipeline (one warp).
// ---------------------------------------------------------------------------
constexpr int N32 = 32;
constexpr int LD = 33;  // padded leading dimension of the warp tile (float2)

// Field of a 16x16 OPD patch embedded at offset 8 in 32x32, then the 2-D
// forward FFT, pruned to the 16 non-zero rows and columns.  On return lane l
// holds F(kx=l, ky=0..31).  opd/amp are the subaperture's 256 values
// (x fastest); tile is the warp's 32x33 float2 scratch.
__device__ __forceinline__ void field_fft_n32(const float* __restrict__ opd, const float* __restrict__ amp,
	float twoinvwvl, float2* tile, int lane, float2 (&F)[32]) {
	// (b) field. lane holds elements e = j*32 + lane: ix = lane&15, iy = 2j + lane/16
	float o[8], a[8];
	float s = 0.f;
#pragma unroll
	for (int j = 0; j < 8; j++) {
		o[j] = __ldg(opd + j * 32 + lane);
		a[j] = __ldg(amp + j * 32 + lane);
		s += o[j];
	}
	// remove the subaperture piston before forming the phase: a constant phase
	// factor cancels in |FFT|^2, and it keeps the FP32 phase small
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
	const float piston = s * (1.f / 256.f);
	const int ix = lane & 15;
#pragma unroll
	for (int j = 0; j < 8; j++) {
		const int iy = 2 * j + (lane >> 4);
		float sn, cs;
		sincospif(twoinvwvl * (o[j] - piston), &sn, &cs);
		tile[iy * LD + ix] = make_float2(a[j] * cs, a[j] * sn);
	}
	__syncwarp();
	// (c) pass along x: lane -> row r=lane&15, half h=lane>>4 (even/odd outputs)
	// X[2m+h] = (-1)^m * (h ? -i : 1) * DFT16(e_j * w32^(h*j))[m]
	{
		const int r = lane & 15, h = lane >> 4;
		float2 e[16];
#pragma unroll
		for (int j = 0; j < 16; j++) e[j] = tile[r * LD + j];
		if (h) twiddle_ramp<-1, 16, 32, 1>(e);
		fft_reg<-1, 16>(e);
		__syncwarp();
#pragma unroll
		for (int m = 0; m < 16; m++) {
			float2 v = e[m];
			if (m & 1) v = make_float2(-v.x, -v.y);
			if (h) v = make_float2(v.y, -v.x);  // * (-i)
			tile[(2 * m + h) * LD + r] = v;      // tile[kx][r]
		}
	}
	__syncwarp();
	// pass along y: lane = kx, 16 inputs at y = 8..23
	{
		float2 c[16], d[16];
#pragma unroll
		for (int j = 0; j < 16; j++) {
			c[j] = tile[lane * LD + j];
			d[j] = c[j];
		}
		twiddle_ramp<-1, 16, 32, 1>(d);
		fft_reg<-1, 16>(c);
		fft_reg<-1, 16>(d);
#pragma unroll
		for (int m = 0; m < 16; m++) {
			float2 v0 = c[m], v1 = d[m];
			if (m & 1) {
				v0 = make_float2(-v0.x, -v0.y);
				v1 = make_float2(-v1.x, -v1.y);
			}
			F[2 * m] = v0;
			F[2 * m + 1] = make_float2(v1.y, -v1.x);
		}
	}
}

// |F|^2 then the forward 2-D FFT of the real PSF. Input: lane = kx holds
// F(kx, ky=0..31).  Output: lane = fy holds OTF(fx=0..31, fy=lane).
__device__ __forceinline__ void psf_to_otf_n32(float2 (&F)[32], float scale, float2* tile, int lane) {
#pragma unroll
	for (int k = 0; k < 32; k++) F[k] = make_float2((F[k].x * F[k].x + F[k].y * F[k].y) * scale, 0.f);
	fft_reg<-1, 32>(F);  // along ky -> Q(kx=lane, fy)
	__syncwarp();
#pragma unroll
	for (int k = 0; k < 32; k++) tile[k * LD + lane] = F[k];  // tile[fy][kx]
	__syncwarp();
#pragma unroll
	for (int k = 0; k < 32; k++) F[k] = tile[lane * LD + k];  // lane = fy
	fft_reg<-1, 32>(F);  // along kx -> OTF(fx, fy=lane)
}

// ---------------------------------------------------------------------------
// LGS uplink OTF (maos/wfsints.c:149-199 with nlwvf == nwvf == notf):
// lotf = FFT(|FFT(embed(lltamp*exp(i*2*pi*lltopd/wvl)))|^2 / nlwvf^2).
// One warp per WFS.  Output transposed: lotfT[fy + 32*fx].
// ---------------------------------------------------------------------------
__global__ void uplink_otf_n32_kernel(const float* const* lltopd, const float* lltamp, float2* const* lotfT,
	int nwfs, float twoinvwvl, float lltnorm) {
	__shared__ float2 tiles[4][32 * LD];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int iw = blockIdx.x * 4 + warp;
	if (iw >= nwfs) return;
	float2 F[32];
	field_fft_n32(lltopd[iw], lltamp, twoinvwvl, tiles[warp], lane, F);
	psf_to_otf_n32(F, lltnorm, tiles[warp], lane);
	float2* out = lotfT[iw];
#pragma unroll
	for (int fx = 0; fx < 32; fx++) out[lane + 32 * fx] = F[fx];
}

// ---------------------------------------------------------------------------
// (e) gradient of one subaperture from its pixel values held by the warp.
// Lane holds pixels p = lane + 32*q.  Sums in FP64.
// ---------------------------------------------------------------------------
template <int NPQ>
__device__ __forceinline__ void grad_from_pixels(const float (&pix)[NPQ], int npix, int pixpsax, int pixpsay,
	const PowfsDev& P, const float* __restrict__ mtche, const float* __restrict__ i0sum, int isa, int lane,
	float* __restrict__ grad, int nsa) {
	if (P.saa && P.saa[isa] < P.saat) return;  // maos/utils.c:1041: vignetted, left unchanged
	double gx = 0, gy = 0;
	if (P.gradtype == 1) {
		// matched filter (maos/utils.c:1043-1060)
		double sx = 0, sy = 0, si = 0;
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) {
				const double v = pix[q];
				sx += (double)__ldg(mtche + 2 * p) * v;
				sy += (double)__ldg(mtche + 2 * p + 1) * v;
				si += v;
			}
		}
#pragma unroll
		for (int off = 16; off > 0; off >>= 1) {
			sx += __shfl_xor_sync(0xffffffffu, sx, off);
			sy += __shfl_xor_sync(0xffffffffu, sy, off);
			si += __shfl_xor_sync(0xffffffffu, si, off);
		}
		double scale = 1.0;
		if (P.sigmatch == 1) {
			scale = (double)i0sum[isa] / si;
			if (scale <= 0 || scale > 10 || !isfinite(scale)) scale = 1;
		}
		gx = sx * scale;
		gy = sy * scale;
	} else {
		// thresholded CoG (math/matmath.c:717-758 via maos/utils.c:1061-1082)
		double sum = 0, sumx = 0, sumy = 0;
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) {
				const double v = (double)pix[q] - (double)P.cogoff;
				if (v > (double)P.cogthres) {
					sum += v;
					sumx += v * (p % pixpsax);
					sumy += v * (p / pixpsax);
				}
			}
		}
#pragma unroll
		for (int off = 16; off > 0; off >>= 1) {
			sum += __shfl_xor_sync(0xffffffffu, sum, off);
			sumx += __shfl_xor_sync(0xffffffffu, sumx, off);
			sumy += __shfl_xor_sync(0xffffffffu, sumy, off);
		}
		double flux = 0;
		if (P.sigmatch == 0) {
			flux = i0sum ? (double)i0sum[isa] : (double)P.sigtot * (P.saa ? P.saa[isa] : 1.f);
		} else if (P.sigmatch == 2) {
			flux = (double)P.sigtot * (P.saa ? P.saa[isa] : 1.f);
		}
		if (flux != 0) sum = flux;
		if (sum > (double)P.cogthres) {
			gx = (sumx / sum - (pixpsax - 1) * 0.5) * P.pixthetax;
			gy = (sumy / sum - (pixpsay - 1) * 0.5) * P.pixthetay;
		}
	}
	if (lane == 0) {
		grad[isa] = (float)gx;
		grad[isa + nsa] = (float)gy;
	}
}

// ---------------------------------------------------------------------------
// (b)-(e) fused, n_opd=16, n_w=n_f=32.  Work item w -> (isa = w / nw, wfs =
// wlist[w % nw]) so the WFS that share a subaperture's ETF run together.
// ---------------------------------------------------------------------------
template <int NPQ>  // pixel slots per lane: ceil(npix/32)
__global__ void __launch_bounds__(128) ints_n32_kernel(PowfsDev P, const WfsDev* __restrict__ wfs, int nw, int nitem) {
	__shared__ float2 tiles[4][32 * LD];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int item = blockIdx.x * 4 + warp;
	if (item >= nitem) return;
	const int isa = item / nw;
	const WfsDev W = wfs[item % nw];
	float2* tile = tiles[warp];
	const size_t off_opd = (size_t)isa * 256;
	float2 F[32];
	field_fft_n32(W.opd + off_opd, W.amp + off_opd, P.twoinvwvl, tile, lane, F);
	psf_to_otf_n32(F, 1.f, tile, lane);
	// lane = fy holds OTF(fx, fy). Uplink OTF (conjugated) and ETF / nominal.
	if (W.lotfT) {
#pragma unroll
		for (int fx = 0; fx < 32; fx++) F[fx] = cmulc(F[fx], __ldg(W.lotfT + lane + 32 * fx));
	}
	if (P.etfT1) {
		const float2* e1 = P.etfT1 + (size_t)isa * 1024 + lane;
		if (P.etfT2) {
			const float2* e2 = P.etfT2 + (size_t)isa * 1024 + lane;
#pragma unroll
			for (int fx = 0; fx < 32; fx++) {
				const float2 a = __ldg(e1 + 32 * fx), b = __ldg(e2 + 32 * fx);
				F[fx] = cmul(F[fx], make_float2(a.x * P.etfwt1 + b.x * P.etfwt2, a.y * P.etfwt1 + b.y * P.etfwt2));
			}
		} else {
#pragma unroll
			for (int fx = 0; fx < 32; fx++) F[fx] = cmul(F[fx], __ldg(e1 + 32 * fx));
		}
	} else if (P.nominalT) {
		const float* nm = P.nominalT + (P.nominal_per_sa ? (size_t)isa * 1024 : 0) + lane;
#pragma unroll
		for (int fx = 0; fx < 32; fx++) {
			const float d = __ldg(nm + 32 * fx);
			F[fx] = make_float2(F[fx].x * d, F[fx].y * d);
		}
	}
	// inverse 2-D FFT, real part: along fx (lane = fy), then along fy (lane = x)
	fft_reg<1, 32>(F);
	__syncwarp();
#pragma unroll
	for (int k = 0; k < 32; k++) tile[k * LD + lane] = F[k];  // tile[x][fy]
	__syncwarp();
#pragma unroll
	for (int k = 0; k < 32; k++) F[k] = tile[lane * LD + k];  // lane = x
	fft_reg<1, 32>(F);
	__syncwarp();
	float* psf = reinterpret_cast<float*>(tile);  // psf[x + 32*y], real part
#pragma unroll
	for (int y = 0; y < 32; y++) psf[lane + 32 * y] = F[y].x;
	__syncwarp();
	// pixel sampling (mkh bilinear map, up to 4 taps per pixel)
	const int npix = P.npix;
	const int* sidx = P.simap_idx + (P.simap_per_sa ? (size_t)isa * npix * 4 : 0);
	const float* swt = P.simap_wt + (P.simap_per_sa ? (size_t)isa * npix * 4 : 0);
	float pix[NPQ];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		float v = 0.f;
		if (p < npix) {
#pragma unroll
			for (int c = 0; c < 4; c++) {
				const int id = __ldg(sidx + 4 * p + c);
				if (id >= 0) v = fmaf(__ldg(swt + 4 * p + c), psf[id], v);
			}
			v *= W.alpha;
		}
		pix[q] = v;
	}
	// (d) noise (lib/libmisc.c:31-55; qe = 1, excess = 1)
	if (W.noisy) {
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) {
				PixelRng rng(W.seed, (uint32_t)(isa * npix + p), W.wfs_id, (uint32_t)P.isim);
				const float tot = pix[q] + P.bkgrnd;
				pix[q] = poisson_draw(rng, tot) + P.rne * rng.normal() - P.bkgrndc;
			}
		}
	}
	if (W.ints) {
		float* o = W.ints + (size_t)isa * npix;
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) o[p] = pix[q];
		}
	}
	if (W.grad) {
		grad_from_pixels<NPQ>(pix, npix, P.pixpsax, P.pixpsay, P, W.mtche + (size_t)isa * 2 * npix,
			W.i0sum, isa, lane, W.grad, P.nsa);
	}
}

// (e) alone: one warp per subaperture from stored intensities.
template <int NPQ>
__global__ void grad_kernel(PowfsDev P, const float* __restrict__ ints, const float* __restrict__ mtche,
	const float* __restrict__ i0sum, float* __restrict__ grad) {
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int isa = blockIdx.x * (blockDim.x >> 5) + warp;
	if (isa >= P.nsa) return;
	float pix[NPQ];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		pix[q] = p < P.npix ? ints[(size_t)isa * P.npix + p] : 0.f;
	}
	grad_from_pixels<NPQ>(pix, P.npix, P.pixpsax, P.pixpsay, P, mtche ? mtche + (size_t)isa * 2 * P.npix : nullptr,
		i0sum, isa, lane, grad, P.nsa);
}

}  // namespace shwfs
