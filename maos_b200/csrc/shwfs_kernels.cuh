// Device kernels of the Shack-Hartmann frame.
//
//   geom_kernel         (a) bilinear gather of every turbulence layer into the
//                           subaperture OPD points of every WFS of the frame
//                           (FP64 offsets), and the LGS uplink OTF
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
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// uniform in [0, 1) with 24-bit resolution
__device__ __forceinline__ float u01(uint32_t v) { return (v >> 8) * (1.0f / 16777216.0f); }
// uniform in (0, 1], for logarithms
__device__ __forceinline__ float u01_nz(uint32_t v) { return ((v >> 8) + 1u) * (1.0f / 16777216.0f); }

// Stream of uniforms for one pixel: counter (n, pixel, wfs, frame).
struct PixelRng {
	uint32_t k0, k1, pix, wfs, frame, n;
	u32x4 buf;
	int used;
	__device__ __forceinline__ PixelRng(uint64_t seed, uint32_t pix_, uint32_t wfs_, uint32_t frame_)
		: k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), pix(pix_), wfs(wfs_), frame(frame_), n(0), used(4) {}
	__device__ __forceinline__ uint32_t bits() {
		if (used == 4) {
			buf = philox4x32_10(u32x4{n++, pix, wfs, frame}, k0, k1);
			used = 0;
		}
		uint32_t v = used == 0 ? buf.x : used == 1 ? buf.y : used == 2 ? buf.z : buf.w;
		used++;
		return v;
	}
	__device__ __forceinline__ float next() { return u01(bits()); }
	// standard normal by Box-Muller: r cos(theta) with theta = pi (2 u2 - 1)
	// uniform on [-pi, pi), the range where the hardware cosine is accurate
	__device__ __forceinline__ float normal() {
		const float u1 = u01_nz(bits()), u2 = next();
		const float r = sqrtf(-2.f * __logf(u1));
		return r * __cosf(3.14159265358979f * fmaf(2.f, u2, -1.f));
	}
};

// Poisson draw of mean xm >= 0.  As the reference (math/random.c:186-209) it
// uses a Gaussian approximation above a mean of 200; below it draws exact
// Poisson variates by another method than the reference's product of
// uniforms (about mean+1 uniforms per draw):
//  - mean < 10: inversion, the smallest k with u < F(k), tested as
//    u e^xm < sum_{j<=k} xm^j / j! so that no small exponential is formed; the
//    walk stops where the next term no longer changes the FP32 sum, beyond
//    which the tail holds less than about 1e-7 of the mass;
//  - 10 <= mean <= 200: transformed rejection with squeeze (W. Hormann, "The
//    transformed rejection method for generating Poisson random variables",
//    Insurance: Mathematics and Economics 12 (1993) 39-45, algorithm PTRS),
//    about 1.1 uniform pairs per draw; the rejection loop is bounded.
struct InvTableF {
	float v[65];
	__host__ __device__ constexpr InvTableF() : v() {
		for (int k = 1; k <= 64; k++) v[k] = 1.0f / (float)k;
	}
};
__constant__ InvTableF c_invkf = InvTableF();

// log(k!) for k < SHWFS_LOGFACT_N, filled from the host (double lgamma,
// rounded) when the first context of a device is created
#define SHWFS_LOGFACT_N 1024
__device__ float g_logfact[SHWFS_LOGFACT_N];
__device__ __forceinline__ float log_factorial(float k) {
	return k < (float)SHWFS_LOGFACT_N ? __ldg(&g_logfact[(int)k]) : lgammaf(k + 1.f);
}

__device__ __forceinline__ float poisson_ptrs(PixelRng& rng, float lam) {
	const float slam = sqrtf(lam), loglam = logf(lam);
	const float b = 0.931f + 2.53f * slam;
	const float a = -0.059f + 0.02483f * b;
	const float invalpha = 1.1239f + 1.1328f / (b - 3.4f);
	const float vr = 0.9277f - 3.6224f / (b - 2.f);
	for (int it = 0; it < 64; it++) {
		const float U = rng.next() - 0.5f, V = rng.next();
		const float us = 0.5f - fabsf(U);
		if (us <= 0.f) continue;  // U = -1/2 exactly: no variate
		const float k = floorf((2.f * a / us + b) * U + lam + 0.43f);
		if (us >= 0.07f && V <= vr) return k;
		if (k < 0.f || (us < 0.013f && V > us)) continue;
		// log V + log(1/alpha) - log(a/us^2 + b) as one logarithm
		if (logf(V * invalpha / (a / (us * us) + b)) <= -lam + k * loglam - log_factorial(k)) return k;
	}
	return rintf(lam);  // 64 rejections in a row: probability below 1e-60
}

__device__ __forceinline__ float poisson_draw(PixelRng& rng, float xm) {
	if (xm > 200.f) return rintf(xm + rng.normal() * sqrtf(xm));
	if (xm >= 10.f) return poisson_ptrs(rng, xm);
	if (!(xm > 0.f)) return 0.f;
	const float t = rng.next() * expf(xm);
	float term = 1.f, S = 1.f;
	int k = 0;
	while (t >= S && k < 64) {
		k++;
		term *= xm * c_invkf.v[k];
		const float S1 = S + term;
		if (S1 == S) break;
		S = S1;
	}
	return (float)k;
}

// ---------------------------------------------------------------------------
// Parameters
// ---------------------------------------------------------------------------
#define SHWFS_MAX_LAYERS 16
#define SHWFS_MAX_ENTRIES 16
#define GEOM_SUM_MAX 32

// One pupil to ray trace in a frame: the subapertures of a WFS, or the LLT
// pupil of an LGS (one "subaperture"), with the per-layer geometry of
// prop_range (lib/accphi.c:241-244) and prop_grid_pts
// (lib/accphi_grid_do.c:424-434), computed on the host in FP64.
struct GeomEntry {
	const double* origx;   // nsa subaperture origins
	const double* origy;
	float* opd;            // nsa*nopd^2 output (may be null for LLT entries)
	int nsa, nopd, item0;  // item0: first block of this entry
	double dx;             // OPD sampling
	double sx[SHWFS_MAX_LAYERS];    // scale / screen dx
	double dispx[SHWFS_MAX_LAYERS]; // (displacement - screen origin) / screen dx
	double dispy[SHWFS_MAX_LAYERS];
	unsigned use;          // bit l: layer l contributes (below the star)
	// LLT entry: uplink OTF (maos/wfsints.c:149-199) written transposed
	const float* lltamp;   // nopd^2, or null for a WFS entry
	float2* lotfT;
	float twoinvwvl, lltnorm;
	// closed-loop and static terms of the pupil's OPD (maos/wfsgrad.c:200-262)
	const float* opdadd;   // nsa*nopd^2 surface added at every point (NCPA), or null
	int has_poly;          // add poly[0] + poly[1] x + poly[2] y + poly[3] (x^2 + y^2) at point (x, y)
	double poly[4];        // tip/tilt, piston and focus terms gathered on the host (FP64)
};
struct GeomParams {
	int nentry, nlayer;
	int interleave;  // items are (subaperture, entry) pairs, entry fastest (all entries have the same nsa)
	// the last nmirror of the nlayer layers are deformable-mirror grids: no wind,
	// no wrap (prop with wrap=0, maos/sim_utils.c:1042; map2loc_linear,
	// cuda/sim/accphi.cu:24-38): a point whose bilinear cell leaves the grid gets
	// nothing from it
	int nmirror;
	// points per thread of the instantiations without a fixed pupil side (0:
	// GEOM_PTS); launches of a few large pupils take 1, for four times the blocks
	int ppt;
	const float* screen[SHWFS_MAX_LAYERS];
	int nx[SHWFS_MAX_LAYERS], ny[SHWFS_MAX_LAYERS];
	float alpha[SHWFS_MAX_LAYERS];
	GeomEntry e[SHWFS_MAX_ENTRIES];
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
	int accum;             // dtrat > 1: add this frame's intensities to the stored ones (maos/wfsints.c)
};

// ---------------------------------------------------------------------------
// Shared pieces of the 32-point pipeline (one warp).
// ---------------------------------------------------------------------------
constexpr int N32 = 32;
constexpr int LD = 33;  // padded leading dimension of the warp tile (float2)

// Field of a 16x16 OPD patch embedded at offset 8 in 32x32, then the 2-D
// forward FFT, pruned to the 16 non-zero rows and columns.  On return lane l
// holds F(kx=l, ky=0..31).  The lane brings the OPD and amplitude of elements
// e = j*32 + lane (ix = lane&15, iy = 2j + lane/16) in o[j], a[j]; tile is
// the warp's 32x33 float2 scratch.
__device__ __forceinline__ void field_fft_n32_regs(const float (&o)[8], const float (&a)[8], float twoinvwvl,
	float2* tile, int lane, float2 (&F)[32]) {
	float s = 0.f;
#pragma unroll
	for (int j = 0; j < 8; j++) s += o[j];
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

// The same with the subaperture's 256 OPD and amplitude values (x fastest)
// read from memory.
__device__ __forceinline__ void field_fft_n32(const float* opd, const float* __restrict__ amp,
	float twoinvwvl, float2* tile, int lane, float2 (&F)[32]) {
	float o[8], a[8];
#pragma unroll
	for (int j = 0; j < 8; j++) {
		o[j] = opd[j * 32 + lane];
		a[j] = amp[j * 32 + lane];
	}
	field_fft_n32_regs(o, a, twoinvwvl, tile, lane, F);
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
// (a) ray trace of every pupil of the frame in one launch (geom_kernel), and
// the LGS uplink OTF of the 32-point path (llt_uplink_kernel): an LLT block
// keeps its OPD in shared memory and its first warp turns it into
// lotf = FFT(|FFT(embed(lltamp*exp(i*2*pi*opd/wvl)))|^2 / nlwvf^2), stored
// transposed (fy fastest).  Item b of geom_kernel belongs to the entry whose
// [item0, item0+nsa) holds it, or, when the launch is interleaved, to entry
// b % nentry at subaperture b / nentry.
// ---------------------------------------------------------------------------
// ---- ray trace (a) ----
// The bilinear coordinates of point (ix, iy) in layer l are separable: the
// column index and weight depend on ix only, the row on iy only.  Each block
// (one subaperture, one OPD point per thread) first tabulates them per layer
// in shared memory: nopd column entries and nopd row entries, each thread
// computing one entry from the FP64 footprint origin (prop_grid_pts,
// lib/accphi_grid_do.c:424-434) with the wrapped neighbour (wrap=1,
// maos/sim_utils.c:1017).  A point then costs two table reads, four gathers
// and the interpolation per layer.  The entries are the same FP32 quantities a
// direct per-point evaluation forms, so the OPD is the same to the bit.
// Dynamic shared memory: nlayer * nopd * 2 * 16 bytes.
//   column entry ix: (jx, jx1, wx, -)      row entry iy: (jy nx, jy1 nx, wy, -)
// A block of bd threads (a multiple of 32, at most 256, chosen so that
// GEOM_PTS * bd covers a pupil with no idle slot where it can) traces up to
// pts * bd points of one subaperture (pts = GEOM_PTS, or GeomParams.ppt);
// larger pupils split each subaperture over bps blocks: block b covers points
// [pts * bd (b % bps), + pts * bd) of subaperture item b / bps.
constexpr int GEOM_PTS = 4;

// The footprint origin of subaperture isa of entry E in layer l along x (isy
// false) or y, in FP64 from the subaperture origin: first screen index j0 and
// FP32 fraction f0, wrapped into the screen (prop_grid_pts,
// lib/accphi_grid_do.c:424-434, wrap=1).
template <bool EXTRA>
__device__ __forceinline__ void geom_origin(const GeomParams& P, const GeomEntry& E, int isa, int l, bool isy, int& j0,
	float& f0) {
	const int n = isy ? P.ny[l] : P.nx[l];
	double x0 = (isy ? E.origy[isa] : E.origx[isa]) * E.sx[l] + (isy ? E.dispy[l] : E.dispx[l]);
	if (!isfinite(x0) || !isfinite((isy ? E.origx[isa] : E.origy[isa]) * E.sx[l] + (isy ? E.dispx[l] : E.dispy[l])))
		x0 = 0;
	if (EXTRA && l >= P.nlayer - P.nmirror) {  // mirror grid: no wrap; the origin may lie off the grid
		x0 = fmin(fmax(x0, -1e9), 1e9);
		j0 = (int)floor(x0);
		f0 = (float)(x0 - j0);
		return;
	}
	x0 -= floor(x0 / n) * n;
	j0 = (int)floor(x0);
	f0 = (float)(x0 - j0);
	if (j0 >= n) j0 -= n;
}
// Point i of a line from its origin (j0, f0) at FP32 step `step` (OPD
// sampling x scale / screen sampling): screen index j, wrapped neighbour j1,
// bilinear weight w.
__device__ __forceinline__ void geom_point(int j0, float f0, int i, float step, int n, int& j, int& j1, float& w) {
	const float f = f0 + i * step;
	const float fl = floorf(f);
	j = j0 + (int)fl;
	while (j >= n) j -= n;
	j1 = j == n - 1 ? 0 : j + 1;
	w = f - fl;
}
// The same on a mirror grid (no wrap): *valid is 0 when the point's cell
// [j, j+1] leaves the grid, and j, j1 are then 0.
__device__ __forceinline__ void geom_point_clip(int j0, float f0, int i, float step, int n, int& j, int& j1, float& w,
	int& valid) {
	const float f = f0 + i * step;
	const float fl = floorf(f);
	j = j0 + (int)fl;
	w = f - fl;
	valid = j >= 0 && j < n - 1;
	if (!valid) j = 0;
	j1 = valid ? j + 1 : 0;
}
// The OPD terms of a pupil point that are not ray traced: the NCPA surface and
// the tip/tilt/piston/focus polynomial (x, y: the point's pupil coordinate).
__device__ __forceinline__ float geom_extra(const GeomEntry& E, int isa, int ipt, int ix, int iy, int np, float acc) {
	if (E.opdadd) acc += E.opdadd[(size_t)isa * np + ipt];
	if (E.has_poly) {
		const double x = E.origx[isa] + ix * E.dx, y = E.origy[isa] + iy * E.dx;
		acc += (float)(E.poly[0] + E.poly[1] * x + E.poly[2] * y + E.poly[3] * (x * x + y * y));
	}
	return acc;
}
// acc + al * bilinear(m00, m10, m01, m11; wx, wy)
__device__ __forceinline__ float geom_bilerp(float al, float m00, float m10, float m01, float m11, float wx, float wy,
	float acc) {
	return fmaf(al, (m00 + (m10 - m00) * wx) * (1.f - wy) + (m01 + (m11 - m01) * wx) * wy, acc);
}

// EXTRA: the launch has mirror grids, NCPA surfaces or polynomial terms (a
// closed-loop frame); the open-loop launch compiles without their code.
// NOPD: the pupil side at compile time (0: the nopd argument; 16 launches
// 64-thread blocks, 32 256-thread blocks); NL: the layer count at compile time
// (0: P.nlayer).
template <bool EXTRA, int NOPD = 0, int NL = 0>
__global__ void __launch_bounds__(NOPD == 16 ? 64 : 256, NOPD == 16 ? 32 : NOPD == 32 ? 8 : 1)
	geom_kernel(const __grid_constant__ GeomParams P, int nopd_arg, int nitem, int bps) {
	const int nopd = NOPD ? NOPD : nopd_arg;
	extern __shared__ int4 s_tab[];
	const int item = blockIdx.x / bps, part = blockIdx.x - item * bps;
	if (item >= nitem) return;
	int ie = 0, isa;
	if (P.interleave) {  // the entries' footprints of one subaperture run together and share L2
		ie = item % P.nentry;
		isa = item / P.nentry;
	} else {
		while (ie + 1 < P.nentry && item >= P.e[ie + 1].item0) ie++;
		isa = item - P.e[ie].item0;
	}
	const GeomEntry& E = P.e[ie];
	const int tid = threadIdx.x, nl = NL ? NL : P.nlayer;
	const int bdim = NOPD == 16 ? 64 : NOPD == 32 ? 256 : (int)blockDim.x;
	// the footprint origin of each (layer, axis) once, in FP64; then the
	// entries of the nopd points of each line from it in FP32
	__shared__ int s_j0[2 * SHWFS_MAX_LAYERS];
	__shared__ float s_f0[2 * SHWFS_MAX_LAYERS], s_step[SHWFS_MAX_LAYERS];
	if (tid < 2 * nl) {
		int j0;
		float f0;
		geom_origin<EXTRA>(P, E, isa, tid >> 1, tid & 1, j0, f0);
		s_j0[tid] = j0;
		s_f0[tid] = f0;
		if (!(tid & 1)) s_step[tid >> 1] = (float)(E.dx * E.sx[tid >> 1]);
	}
	__syncthreads();
	for (int k = tid; k < nl * 2 * nopd; k += bdim) {
		const int l = k / (2 * nopd), r = k - l * 2 * nopd;
		const bool isy = r >= nopd;
		const int i = isy ? r - nopd : r;
		const int n = isy ? P.ny[l] : P.nx[l];
		int j, j1, valid = 1;
		float w;
		if (!EXTRA || l < nl - P.nmirror)
			geom_point(s_j0[2 * l + isy], s_f0[2 * l + isy], i, s_step[l], n, j, j1, w);
		else
			geom_point_clip(s_j0[2 * l + isy], s_f0[2 * l + isy], i, s_step[l], n, j, j1, w, valid);
		const int m = isy ? P.nx[l] : 1;
		s_tab[k] = make_int4(j * m, j1 * m, __float_as_int(w), valid);
	}
	__syncthreads();
	// up to GEOM_PTS points per thread, layers outermost so that the gathers of the points are in flight
	// together; every point still sums its layers in order
	const int bd = bdim;
	const int pts = NOPD || P.ppt <= 0 || P.ppt > GEOM_PTS ? GEOM_PTS : P.ppt;
	const int np = nopd * nopd, p0 = pts * bd * part, p1 = min(np, p0 + pts * bd);
	float acc[GEOM_PTS];
	int ixu[GEOM_PTS], iyu[GEOM_PTS];
#pragma unroll
	for (int u = 0; u < GEOM_PTS; u++) {
		const int ip = p0 + tid + bd * u;
		acc[u] = 0.f;
		ixu[u] = ip % nopd;
		iyu[u] = ip / nopd;
	}
	const int nwrap = EXTRA ? nl - P.nmirror : nl;
	// 16x16 and 32x32 pupils: a thread's points fill whole rows of one column
	// (64 or 256 threads, four rows apart), so they share the column entry and
	// need no bounds test
	constexpr bool ONECOL = NOPD == 16 || NOPD == 32;
#pragma unroll
	for (int l = 0; l < nwrap; l++) {
		if (!((E.use >> l) & 1u)) continue;
		const float* __restrict__ sc = P.screen[l];
		const float al = P.alpha[l];
		const int4 tx0 = s_tab[l * 2 * nopd + ixu[0]];
#pragma unroll
		for (int u = 0; u < GEOM_PTS; u++) {
			if (ONECOL || p0 + tid + bd * u < p1) {
				const int4 tx = ONECOL ? tx0 : s_tab[l * 2 * nopd + ixu[u]], ty = s_tab[l * 2 * nopd + nopd + iyu[u]];
				const float m00 = __ldg(sc + (ty.x + tx.x)), m10 = __ldg(sc + (ty.x + tx.y));
				const float m01 = __ldg(sc + (ty.y + tx.x)), m11 = __ldg(sc + (ty.y + tx.y));
				acc[u] = geom_bilerp(al, m00, m10, m01, m11, __int_as_float(tx.z), __int_as_float(ty.z), acc[u]);
			}
		}
	}
	for (int l = nwrap; EXTRA && l < nl; l++) {  // mirror grids: only points whose cell lies on the grid and is valid
		if (!((E.use >> l) & 1u)) continue;
		const float* __restrict__ sc = P.screen[l];
		const float al = P.alpha[l];
#pragma unroll
		for (int u = 0; u < GEOM_PTS; u++) {
			if (p0 + tid + bd * u < p1) {
				const int4 tx = s_tab[l * 2 * nopd + ixu[u]], ty = s_tab[l * 2 * nopd + nopd + iyu[u]];
				if (tx.w & ty.w) {
					const float m00 = __ldg(sc + (ty.x + tx.x)), m10 = __ldg(sc + (ty.x + tx.y));
					const float m01 = __ldg(sc + (ty.y + tx.x)), m11 = __ldg(sc + (ty.y + tx.y));
					const float wx = __int_as_float(tx.z), wy = __int_as_float(ty.z);
					const float v = (m00 + (m10 - m00) * wx) * (1.f - wy) + (m01 + (m11 - m01) * wx) * wy;
					// NaN marks grid points outside the mirror (add_valid, math/numtype.h:40)
					if (!isnan(v)) acc[u] = fmaf(al, v, acc[u]);
				}
			}
		}
	}
	if (EXTRA && (E.opdadd || E.has_poly)) {
#pragma unroll
		for (int u = 0; u < GEOM_PTS; u++)
			if (p0 + tid + bd * u < p1) acc[u] = geom_extra(E, isa, p0 + tid + bd * u, ixu[u], iyu[u], np, acc[u]);
	}
#pragma unroll
	for (int u = 0; u < GEOM_PTS; u++)
		if (p0 + tid + bd * u < p1) E.opd[(size_t)isa * np + p0 + tid + bd * u] = acc[u];
}

// LGS uplink: ray trace of each LLT pupil (one block of 256 threads per
// pupil, nopd == 16) into shared memory, then its first warp forms the
// uplink OTF.  Runs beside geom_kernel on a second stream.
__global__ void __launch_bounds__(256) llt_uplink_kernel(const __grid_constant__ GeomParams P) {
	__shared__ float s_opd[256];
	__shared__ float2 s_tile[32 * LD];
	__shared__ int s_i0[SHWFS_MAX_LAYERS][2];
	__shared__ float s_f0[SHWFS_MAX_LAYERS][3];  // x fraction, y fraction, step
	const GeomEntry& E = P.e[blockIdx.x];
	const int ip = threadIdx.x;
	const int ix = ip & 15, iy = ip >> 4;
	// the pupil's FP64 origin in each layer once (thread l), -1 where it is not finite
	if (ip < P.nlayer - P.nmirror) {
		const int l = ip, nx = P.nx[l], ny = P.ny[l];
		double x0 = E.origx[0] * E.sx[l] + E.dispx[l];
		double y0 = E.origy[0] * E.sx[l] + E.dispy[l];
		if (!isfinite(x0) || !isfinite(y0)) {
			s_i0[l][0] = -1;
		} else {
			x0 -= floor(x0 / nx) * nx;
			y0 -= floor(y0 / ny) * ny;
			const int ix0 = (int)floor(x0), iy0 = (int)floor(y0);
			s_i0[l][0] = ix0;
			s_i0[l][1] = iy0;
			s_f0[l][0] = (float)(x0 - ix0);
			s_f0[l][1] = (float)(y0 - iy0);
			s_f0[l][2] = (float)(E.dx * E.sx[l]);
		}
	}
	__syncthreads();
	float acc = 0.f;
	for (int l = 0; l < P.nlayer - P.nmirror; l++) {
		if (!((E.use >> l) & 1u) || s_i0[l][0] < 0) continue;
		const int nx = P.nx[l], ny = P.ny[l];
		const int ix0 = s_i0[l][0], iy0 = s_i0[l][1];
		const float step = s_f0[l][2];
		const float xf = s_f0[l][0] + ix * step, yf = s_f0[l][1] + iy * step;
		const float flx = floorf(xf), fly = floorf(yf);
		int jx = ix0 + (int)flx, jy = iy0 + (int)fly;
		const float wx = xf - flx, wy = yf - fly;
		while (jx >= nx) jx -= nx;
		while (jy >= ny) jy -= ny;
		const int jx1 = jx == nx - 1 ? 0 : jx + 1, jy1 = jy == ny - 1 ? 0 : jy + 1;
		const float* sc = P.screen[l];
		const float m00 = __ldg(sc + jx + (size_t)nx * jy), m10 = __ldg(sc + jx1 + (size_t)nx * jy);
		const float m01 = __ldg(sc + jx + (size_t)nx * jy1), m11 = __ldg(sc + jx1 + (size_t)nx * jy1);
		acc += P.alpha[l] * ((m00 + (m10 - m00) * wx) * (1.f - wy) + (m01 + (m11 - m01) * wx) * wy);
	}
	if (E.has_poly) acc = geom_extra(E, 0, ip, ix, iy, 256, acc);  // uplink tip/tilt (maos/wfsgrad.c:373-377)
	s_opd[ip] = acc;
	if (E.opd) E.opd[ip] = acc;
	__syncthreads();
	if (ip < 32) {
		float2 F[32];
		field_fft_n32(s_opd, E.lltamp, E.twoinvwvl, s_tile, ip, F);
		psf_to_otf_n32(F, E.lltnorm, s_tile, ip);
#pragma unroll
		for (int fx = 0; fx < 32; fx++) E.lotfT[ip + 32 * fx] = F[fx];
	}
}

// Uplink OTF from a given LLT OPD (one warp per WFS), for callers that hold
// the LLT OPD already (shwfs_ints_grad_dev).
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
// s2 serves sigmatch 2 (normalisation by the whole frame's intensity,
// maos/utils.c:1013-1036): the matched filter's scale i0sumg / i1sum, or the
// CoG's signal level i1sum / saasum; unused otherwise.
__device__ __forceinline__ void grad_from_pixels(const float (&pix)[NPQ], int npix, int pixpsax, int pixpsay,
	const PowfsDev& P, const float* __restrict__ mtche, const float* __restrict__ i0sum, int isa, int lane,
	float* __restrict__ grad, int nsa, double s2 = 0) {
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
		} else if (P.sigmatch == 2) {
			scale = s2;
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
			flux = s2 * (P.saa ? P.saa[isa] : 1.f);
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
template <int NPQ>
__device__ __forceinline__ void ints_n32_pixels(const PowfsDev& P, const WfsDev& W, int isa, int lane,
	const float* psf);

// (c)-(e) of one subaperture image after its field transform: F from
// field_fft_n32 (lane = kx holds F(kx, ky=0..31)); tile is the warp's scratch.
template <int NPQ>
__device__ __forceinline__ void ints_n32_tail(const PowfsDev& P, const WfsDev& W, int isa, int lane, float2* tile,
	float2 (&F)[32]) {
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
	ints_n32_pixels<NPQ>(P, W, isa, lane, psf);
}

// (c)-(e) after the image is in shared memory (psf[x + 32 y], the real part of
// the inverse transform): pixel sampling, noise, stored intensities, gradients.
template <int NPQ>
__device__ __forceinline__ void ints_n32_pixels(const PowfsDev& P, const WfsDev& W, int isa, int lane,
	const float* psf) {
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
			if (P.accum) v += W.ints[(size_t)isa * npix + p];  // dtrat > 1: the frames so far
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

// ---- half-spectrum form of (c): the PSF is real, so its OTF is formed only
// for fy = 0..16 and the image comes back through a complex-to-real inverse.
// The columns fy = 0 and 16 (real along ky) travel packed as one complex
// column, so 16 spectral columns remain, and lanes c and c + 16 share column
// c: each does a 16-point transform of the even (c) or odd (c + 16) samples
// and one exchange of 8 values forms the 32-point column.  Per image this is
// four 16-point transforms per lane where the full spectrum takes four
// 32-point ones, with half the transfer-function products.  The transfer
// function (uplink OTF, ETF or DTF nominal: transforms of real kernels) is
// Hermitian, so the half spectrum carries the whole product; the image equals
// the real part of the full inverse (maos/wfsints.c:284-286 takes that real
// part) up to rounding.

// X[k] = sum_n x[n] w32^(kn), k = 0..16, of the real x held as z[n] = x[2n] +
// i x[2n+1] after z = FFT16(z): X[0] and X[16] (real) packed as Q[0] = (X0,
// X16), Q[k] = X[k] for k = 1..15.
template <int K>
__device__ __forceinline__ void r2c32_post(const float2 (&z)[16], float2 (&Q)[16]) {
	if constexpr (K < 16) {
		const float2 a = z[K], b = make_float2(z[16 - K].x, -z[16 - K].y);
		const float2 sm = cadd(a, b), df = csub(a, b);
		const float2 t = twmul<-1, 32, K>(make_float2(df.y, -df.x));  // w^K * (-i) * (a - b)
		Q[K] = make_float2(0.5f * (sm.x + t.x), 0.5f * (sm.y + t.y));
		r2c32_post<K + 1>(z, Q);
	}
}
// The inverse: Z[k] = (Y[k] + Y[k+16]) + i w32^(-k) (Y[k] - Y[k+16]) with
// Y[k+16] = conj Y[16-k], so that IFFT16(Z)[n] = y[2n] + i y[2n+1] for the
// real y[n] = sum_k Y[k] w32^(-kn) of the Hermitian Y (Y[0], Y[16] packed).
template <int K>
__device__ __forceinline__ void c2r32_pre(const float2 (&Y)[16], float2 (&Z)[16]) {
	if constexpr (K < 16) {
		const float2 a = Y[K], b = make_float2(Y[16 - K].x, -Y[16 - K].y);
		const float2 sm = cadd(a, b);
		const float2 t = twmul<1, 32, K>(csub(a, b));
		Z[K] = make_float2(sm.x - t.y, sm.y + t.x);
		c2r32_pre<K + 1>(Y, Z);
	}
}
// i * w32^(-k) (v) for k = i + 8h: the compile-time part w32^(-i), then i^h
template <int I>
__device__ __forceinline__ void inv_ramp8(float2 (&v)[8], int h) {
	if constexpr (I < 8) {
		float2 t = twmul<1, 32, I>(v[I]);
		if (h) t = make_float2(-t.y, t.x);
		v[I] = t;
		inv_ramp8<I + 1>(v, h);
	}
}
// v[i] times the transfer function at element e0 + stride*i (fx*32 + fy of
// the transposed arrays): conj(uplink OTF) x (ETF, the blend of two ETFs, or
// the DTF nominal).  The conditions are uniform over the warp and each
// factor's NV loads are issued together.
template <int NV>
__device__ __forceinline__ void tf_apply(const PowfsDev& P, const WfsDev& W, int isa, int e0, int stride,
	float2 (&v)[NV]) {
	if (W.lotfT) {
		float2 l[NV];
#pragma unroll
		for (int i = 0; i < NV; i++) l[i] = __ldg(W.lotfT + e0 + stride * i);
#pragma unroll
		for (int i = 0; i < NV; i++) v[i] = cmulc(v[i], l[i]);
	}
	if (P.etfT1) {
		const float2* e1 = P.etfT1 + (size_t)isa * 1024 + e0;
		float2 a[NV];
#pragma unroll
		for (int i = 0; i < NV; i++) a[i] = __ldg(e1 + stride * i);
		if (P.etfT2) {
			const float2* e2 = P.etfT2 + (size_t)isa * 1024 + e0;
#pragma unroll
			for (int i = 0; i < NV; i++) {
				const float2 b = __ldg(e2 + stride * i);
				a[i] = make_float2(a[i].x * P.etfwt1 + b.x * P.etfwt2, a[i].y * P.etfwt1 + b.y * P.etfwt2);
			}
		}
#pragma unroll
		for (int i = 0; i < NV; i++) v[i] = cmul(v[i], a[i]);
	} else if (P.nominalT) {
		const float* nm = P.nominalT + (P.nominal_per_sa ? (size_t)isa * 1024 : 0) + e0;
		float d[NV];
#pragma unroll
		for (int i = 0; i < NV; i++) d[i] = __ldg(nm + stride * i);
#pragma unroll
		for (int i = 0; i < NV; i++) v[i] = make_float2(v[i].x * d[i], v[i].y * d[i]);
	}
}

// F from field_fft_n32 (lane = kx holds F(kx, ky=0..31)) -> psf[x + 32 y] in
// tile, the real image before pixel sampling.
__device__ __forceinline__ void otf_tf_inverse_half_n32(const PowfsDev& P, const WfsDev& W, int isa, int lane,
	float2* tile, const float2 (&F)[32]) {
	// PSF row kx = lane along ky as 16 complex pairs, then its real FFT
	float2 Q[16];
	{
		float2 z[16];
#pragma unroll
		for (int n = 0; n < 16; n++)
			z[n] = make_float2(F[2 * n].x * F[2 * n].x + F[2 * n].y * F[2 * n].y,
				F[2 * n + 1].x * F[2 * n + 1].x + F[2 * n + 1].y * F[2 * n + 1].y);
		fft_reg<-1, 16>(z);
		Q[0] = make_float2(z[0].x + z[0].y, z[0].x - z[0].y);
		r2c32_post<1>(z, Q);
	}
	__syncwarp();
#pragma unroll
	for (int c = 0; c < 16; c++) tile[c * LD + lane] = Q[c];  // tile[c][kx]
	__syncwarp();
	// column c = lane & 15 along kx: h = 0 the even kx, h = 1 the odd kx
	const int c = lane & 15, h = lane >> 4;
	float2 A[8], B[8];  // G(fx) at fx = i + 8h (A) and i + 8h + 16 (B)
	{
		float2 v[16];
#pragma unroll
		for (int j = 0; j < 16; j++) v[j] = tile[c * LD + 2 * j + h];
		fft_reg<-1, 16>(v);
		if (h) twiddle_ramp<-1, 16, 32, 1>(v);  // w^k O[k]
#pragma unroll
		for (int i = 0; i < 8; i++) {
			const float2 sd = h ? v[i] : v[8 + i];
			const float2 r = make_float2(__shfl_xor_sync(0xffffffffu, sd.x, 16), __shfl_xor_sync(0xffffffffu, sd.y, 16));
			const float2 ev = h ? r : v[i], od = h ? v[8 + i] : r;
			A[i] = cadd(ev, od);
			B[i] = csub(ev, od);
		}
	}
	// column 0 holds Gp = G(fx, 0) + i G(fx, 16), both Hermitian in fx.  Lanes
	// 0 and 16 put it in a scratch row; every lane then splits one fx with the
	// mirrored value Gp(-fx), applies the transfer function at fy = 0 and 16,
	// and packs the products again in a second row, which lanes 0 and 16 take
	// back after the other columns' products.
	float2* scr = tile + 16 * LD;
	float2* scr2 = tile + 17 * LD;
	if (c == 0) {
#pragma unroll
		for (int i = 0; i < 8; i++) {
			scr[i + 8 * h] = A[i];
			scr[i + 8 * h + 16] = B[i];
		}
	}
	__syncwarp();
	{
		const float2 g = scr[lane], m = scr[(32 - lane) & 31];
		float2 y0[1] = {make_float2(0.5f * (g.x + m.x), 0.5f * (g.y - m.y))};
		float2 y16[1] = {make_float2(0.5f * (g.y + m.y), -0.5f * (g.x - m.x))};
		tf_apply<1>(P, W, isa, lane * 32, 0, y0);
		tf_apply<1>(P, W, isa, lane * 32 + 16, 0, y16);
		scr2[lane] = make_float2(y0[0].x - y16[0].y, y0[0].y + y16[0].x);
	}
	tf_apply<8>(P, W, isa, 8 * h * 32 + c, 32, A);
	tf_apply<8>(P, W, isa, (8 * h + 16) * 32 + c, 32, B);
	__syncwarp();
	if (c == 0) {
#pragma unroll
		for (int i = 0; i < 8; i++) {
			A[i] = scr2[i + 8 * h];
			B[i] = scr2[i + 8 * h + 16];
		}
	}
	// inverse along fx: h = 0 forms the even x, h = 1 the odd x
	float2 X[16];
	{
		float2 u[8], d[8];
#pragma unroll
		for (int i = 0; i < 8; i++) {
			u[i] = cadd(A[i], B[i]);
			d[i] = csub(A[i], B[i]);
		}
		inv_ramp8<0>(d, h);
#pragma unroll
		for (int i = 0; i < 8; i++) {
			const float2 sd = h ? u[i] : d[i];
			const float2 r = make_float2(__shfl_xor_sync(0xffffffffu, sd.x, 16), __shfl_xor_sync(0xffffffffu, sd.y, 16));
			X[i] = h ? r : u[i];
			X[8 + i] = h ? d[i] : r;
		}
		fft_reg<1, 16>(X);  // y(x = 2m + h, c)
	}
	__syncwarp();
#pragma unroll
	for (int m = 0; m < 16; m++) tile[(2 * m + h) * LD + c] = X[m];  // tile[x][c]
	__syncwarp();
	// row x = lane along fy: complex-to-real
	{
		float2 Y[16], Z[16];
#pragma unroll
		for (int k = 0; k < 16; k++) Y[k] = tile[lane * LD + k];
		Z[0] = make_float2(Y[0].x + Y[0].y, Y[0].x - Y[0].y);
		c2r32_pre<1>(Y, Z);
		fft_reg<1, 16>(Z);
		__syncwarp();
		float* psf = reinterpret_cast<float*>(tile);
#pragma unroll
		for (int n = 0; n < 16; n++) {
			psf[lane + 64 * n] = Z[n].x;
			psf[lane + 64 * n + 32] = Z[n].y;
		}
	}
	__syncwarp();
}

template <int NPQ>
__device__ __forceinline__ void ints_n32_tail_half(const PowfsDev& P, const WfsDev& W, int isa, int lane,
	float2* tile, const float2 (&F)[32]) {
	otf_tf_inverse_half_n32(P, W, isa, lane, tile, F);
	ints_n32_pixels<NPQ>(P, W, isa, lane, reinterpret_cast<const float*>(tile));
}

// NPQ: pixel slots per lane, ceil(npix/32).  MINB: resident blocks per SM the
// register allocation must allow (occupancy/spill trade-off, picked by the
// autotuner).  HALF: the half-spectrum form of (c).
template <int NPQ, int MINB, bool HALF = false>
__global__ void __launch_bounds__(128, MINB) ints_n32_kernel(PowfsDev P, const WfsDev* __restrict__ wfs, int nw, int nitem) {
	__shared__ float2 tiles[4][32 * LD];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int item = blockIdx.x * 4 + warp;
	if (item >= nitem) return;
	const int isa = item / nw;
	const WfsDev W = wfs[item % nw];
	float2* tile = tiles[warp];
	const size_t off_opd = (size_t)isa * 256;
	float2 F[32];
	// the subaperture's ETF (8 KB, read after the first two transforms) into L2 now
	if (P.etfT1) {
		prefetch_l2(P.etfT1 + (size_t)isa * 1024 + 32 * lane);
		prefetch_l2(P.etfT1 + (size_t)isa * 1024 + 32 * lane + 16);
	}
	field_fft_n32(W.opd + off_opd, W.amp + off_opd, P.twoinvwvl, tile, lane, F);
	if (HALF) ints_n32_tail_half<NPQ>(P, W, isa, lane, tile, F);
	else ints_n32_tail<NPQ>(P, W, isa, lane, tile, F);
}

// (d)-(e) after an imaging kernel that stored noise-free intensities (the
// tensor-core form): photon/read noise in place, then CoG / matched filter.
// One warp per work item, items ordered as in the imaging launch.
template <int NPQ>
__global__ void noise_grad_kernel(PowfsDev P, const WfsDev* __restrict__ wfs, int nw, int nitem) {
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int item = blockIdx.x * (blockDim.x >> 5) + warp;
	if (item >= nitem) return;
	const int isa = item / nw;
	const WfsDev& W = wfs[item % nw];
	const int npix = P.npix;
	float* o = W.ints + (size_t)isa * npix;
	float pix[NPQ];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		pix[q] = p < npix ? o[p] : 0.f;
	}
	if (W.noisy) {
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) {
				PixelRng rng(W.seed, (uint32_t)(isa * npix + p), W.wfs_id, (uint32_t)P.isim);
				pix[q] = poisson_draw(rng, pix[q] + P.bkgrnd) + P.rne * rng.normal() - P.bkgrndc;
				o[p] = pix[q];
			}
		}
	}
	if (W.grad)
		grad_from_pixels<NPQ>(pix, npix, P.pixpsax, P.pixpsay, P, W.mtche + (size_t)isa * 2 * npix, W.i0sum, isa,
			lane, W.grad, P.nsa);
}

// Noise of geometric gradients, add_geom_noise_do (cuda/sim/wfsgrad.cu:39-51):
// nea holds per subaperture the lower Cholesky factor (xx, yy, xy) of the
// gradient noise covariance; gx += n1 nea_xx, gy += n2 nea_yy + n1 nea_xy,
// n1 and n2 standard normals from the Philox stream (seed, 2^31 + isa, wfs,
// frame).
__device__ __forceinline__ void geom_noise(float& gx, float& gy, int isa, int nsa, const float* __restrict__ nea,
	uint64_t seed, uint32_t wfs_id, uint32_t frame) {
	PixelRng rng(seed, 0x80000000u + (uint32_t)isa, wfs_id, frame);
	const float n1 = rng.normal(), n2 = rng.normal();
	gx = fmaf(n1, nea[isa], gx);
	gy = fmaf(n2, nea[isa + nsa], fmaf(n1, nea[isa + 2 * nsa], gy));
}

// Geometric gradients (z-tilt): the amplitude-weighted least-squares plane
// of each subaperture's OPD, as cuztilt_do (cuda/sim/wfsgrad.cu:57-106) with
// the inverse moment matrix of pts_mcc_ptt (math/loc.c:612-650) formed here:
// g = [(b0, b1, b2) . imcc(:, 1), (b0, b1, b2) . imcc(:, 2)], b = (sum a o,
// sum a o x, sum a o y), imcc = inv(sum a [1 x y]'[1 x y]), x = origx + ix dx.
// One warp per subaperture, FP64 sums; with nea, geom_noise is added.
__global__ void ztilt_kernel(const float* __restrict__ opd, const float* __restrict__ amp,
	const double* __restrict__ origx, const double* __restrict__ origy, int nsa, int nopd, double dx,
	float* __restrict__ grad, const float* __restrict__ nea, uint64_t seed, uint32_t wfs_id, uint32_t frame) {
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int isa = blockIdx.x * (blockDim.x >> 5) + warp;
	if (isa >= nsa) return;
	const int np = nopd * nopd;
	const double ox = origx[isa], oy = origy[isa];
	double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // a00 a01 a02 a11 a12 a22 b0 b1 b2
	for (int ip = lane; ip < np; ip += 32) {
		const double x = ox + (ip % nopd) * dx, y = oy + (ip / nopd) * dx;
		const double a = amp[(size_t)isa * np + ip], ao = a * (double)opd[(size_t)isa * np + ip];
		m[0] += a;
		m[1] += a * x;
		m[2] += a * y;
		m[3] += a * x * x;
		m[4] += a * x * y;
		m[5] += a * y * y;
		m[6] += ao;
		m[7] += ao * x;
		m[8] += ao * y;
	}
#pragma unroll
	for (int k = 0; k < 9; k++)
#pragma unroll
		for (int off = 16; off > 0; off >>= 1) m[k] += __shfl_xor_sync(0xffffffffu, m[k], off);
	if (lane == 0) {
		const double a00 = m[0], a01 = m[1], a02 = m[2], a11 = m[3], a12 = m[4], a22 = m[5];
		// inverse of the symmetric 3x3 by cofactors
		const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
		const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
		const double det = a00 * c00 + a01 * c01 + a02 * c02;
		float gx = 0.f, gy = 0.f;
		if (det != 0) {
			gx = (float)((m[6] * c01 + m[7] * c11 + m[8] * c12) / det);
			gy = (float)((m[6] * c02 + m[7] * c12 + m[8] * c22) / det);
		}
		if (nea) geom_noise(gx, gy, isa, nsa, nea, seed, wfs_id, frame);
		grad[isa] = gx;
		grad[isa + nsa] = gy;
	}
}

// Geometric gradients (G-tilt): grad = GS0 opd, GS0 the averaged-gradient
// operator of mkg (lib/mkg.c:471-477) held in CSR (2 nsa rows, nsa nopd^2
// columns), as cuspmul in cuda/sim/wfsgrad.cu:649.  One warp per
// subaperture (rows isa and isa + nsa), FP64 sums; noise as ztilt_kernel.
__global__ void gtilt_kernel(const int* __restrict__ rowptr, const int* __restrict__ col,
	const float* __restrict__ val, int nsa, const float* __restrict__ opd, float* __restrict__ grad,
	const float* __restrict__ nea, uint64_t seed, uint32_t wfs_id, uint32_t frame) {
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int isa = blockIdx.x * (blockDim.x >> 5) + warp;
	if (isa >= nsa) return;
	double sx = 0, sy = 0;
	for (int k = rowptr[isa] + lane, e = rowptr[isa + 1]; k < e; k += 32) sx += (double)val[k] * opd[col[k]];
	for (int k = rowptr[isa + nsa] + lane, e = rowptr[isa + nsa + 1]; k < e; k += 32)
		sy += (double)val[k] * opd[col[k]];
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) {
		sx += __shfl_xor_sync(0xffffffffu, sx, off);
		sy += __shfl_xor_sync(0xffffffffu, sy, off);
	}
	if (lane == 0) {
		float gx = (float)sx, gy = (float)sy;
		if (nea) geom_noise(gx, gy, isa, nsa, nea, seed, wfs_id, frame);
		grad[isa] = gx;
		grad[isa + nsa] = gy;
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

// sigmatch 2: the total intensity of each WFS of a launch (i1sum,
// maos/utils.c:1022-1026), FP64; grid (blocks, nw), sums zeroed before.
struct SumParams {
	int nw;
	long n;                          // intensities per WFS
	const float* ints[GEOM_SUM_MAX];
	double* sum[GEOM_SUM_MAX];
};
__global__ void ints_sum_kernel(const __grid_constant__ SumParams S) {
	const int k = blockIdx.y;
	const float* x = S.ints[k];
	double t = 0;
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += (long)gridDim.x * blockDim.x) t += x[i];
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
	__shared__ double red[32];
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
	__syncthreads();
	if (threadIdx.x == 0) {
		double u = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) u += red[w];
		atomicAdd(S.sum[k], u);
	}
}

// sigmatch 2 gradients of one WFS from its stored intensities once i1sum is
// known: s2 = i0sumg / i1sum (matched filter) or i1sum / saasum (CoG).
template <int NPQ>
__global__ void grad_sig2_kernel(PowfsDev P, const float* __restrict__ ints, const float* __restrict__ mtche,
	const float* __restrict__ i0sum, float* __restrict__ grad, const double* __restrict__ i1sum, double i0sumg,
	double saasum) {
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int isa = blockIdx.x * (blockDim.x >> 5) + warp;
	if (isa >= P.nsa) return;
	const double s2 = P.gradtype == 1 ? i0sumg / *i1sum : *i1sum / saasum;
	float pix[NPQ];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		pix[q] = p < P.npix ? ints[(size_t)isa * P.npix + p] : 0.f;
	}
	grad_from_pixels<NPQ>(pix, P.npix, P.pixpsax, P.pixpsay, P, mtche ? mtche + (size_t)isa * 2 * P.npix : nullptr,
		i0sum, isa, lane, grad, P.nsa, s2);
}

// Photon and read noise on n intensities in place, the rule of addnoise
// (lib/libmisc.c:31-55): tot = x + bkgrnd + bkgrnd2[i], times qe[i] when
// given; x = (Poisson(tot excess) + tot (1 - excess) + rne N(0,1)) qe[i]
// - (bkgrndc + bkgrnd2c[i]).  Draws come from the counter (seed, i, stream, frame).
__global__ void addnoise_kernel(float* __restrict__ x, long n, const float* __restrict__ bkgrnd2,
	const float* __restrict__ bkgrnd2c, const float* __restrict__ qe, float bkgrnd, float bkgrndc, float rne,
	float excess, uint64_t seed, uint32_t stream, uint32_t frame) {
	for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
		float tot = x[i] + bkgrnd + (bkgrnd2 ? bkgrnd2[i] : 0.f);
		const float corr = bkgrndc + (bkgrnd2c ? bkgrnd2c[i] : 0.f);
		float scale = 1.f;
		if (qe) {
			tot *= qe[i];
			scale = 1.f / qe[i];
		}
		PixelRng rng(seed, (uint32_t)i, stream, frame);
		const float ph = poisson_draw(rng, tot * excess);
		x[i] = (ph + tot * (1.f - excess) + rne * rng.normal()) / scale - corr;
	}
}

}  // namespace shwfs
