// Imaging stages (b)-(e) for the larger FFT sizes, n_f = n_w = N in {64, 128,
// 256} (the NGS and tip-tilt sensors of an uneven batch, large-sampling LGS):
// a chain of batched 1-D FFT passes over a per-powfs scratch image in global
// memory (L2-resident for the small batches), each pass a kernel that moves
// tiles of 16 rows or 16 columns of an image through shared memory, with the
// element-wise step of the chain fused in:
//
//   pass 1  rows y in [pad, pad+n_o):   field E = amp exp(i 2 pi opd / lambda), FFT along x
//   pass 2  columns kx:                 FFT along y (rows outside the pupil are zero), |.|^2 * scale
//   pass 3  rows ky:                    FFT along kx
//   pass 4  columns fx:                 FFT along ky, x conj(uplink OTF) x ETF / DTF nominal
//   pass 5  rows fy:                    inverse FFT along fx
//   pass 6  columns x:                  inverse FFT along fy, real part
//   pixels  one warp per image:         bilinear pixel map, noise, CoG / matched filter
//
// as maos/wfsints.c:233-286 (cembed_wvf with pad (n_w - n_o)/2, cfft2 with
// FFTW's sign and no normalisation, cabs2toreal, ccwmc with the uplink OTF,
// apply_dtf_etf, cfft2 inverse, dspmulcreal).  For the LLT pupil, passes 1-4
// without a transfer function give the uplink OTF (maos/wfsints.c:149-199).
// Transfer functions are stored transposed per subaperture ([fy + N fx]), as
// in the 32-point path; the scratch image is row-major ([row][column]).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "shwfs_kernels.cuh"

namespace shwfs {

// FFT lines per tile: 16 (128-byte row segments in the column passes), fewer
// for the large transforms of the small batches, for more blocks
__host__ __device__ constexpr int gen_lines(int n) { return n >= 256 ? 4 : n >= 128 ? 8 : 16; }
constexpr int GEN_THREADS = 256;

enum GenPass { GEN_FIELD_ROWS = 1, GEN_PSF_COLS, GEN_OTF_ROWS, GEN_OTF_COLS, GEN_INV_ROWS, GEN_INV_COLS };

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// In-place radix-2 FFT of gen_lines(N) lines of N points in shared memory, line
// stride N + 1 (bank-conflict free for column tiles), input in bit-reversed
// order.  tw[k] = exp(-2 pi i k / N), k < N/2; dir -1 forward, +1 inverse.
template <int N>
__device__ __forceinline__ void fft_lines(float2* s, const float2* __restrict__ tw, int dir) {
	constexpr int LOGN = ilog2c(N), LS = N + 1, NB = gen_lines(N) * N / 2;
#pragma unroll 1
	for (int st = 0; st < LOGN; st++) {
		const int half = 1 << st;
		for (int b = threadIdx.x; b < NB; b += GEN_THREADS) {
			const int line = b / (N / 2), j = b - line * (N / 2);
			const int grp = j >> st, pos = j & (half - 1);
			const int k0 = grp * 2 * half + pos, k1 = k0 + half;
			float2 w = tw[pos << (LOGN - 1 - st)];
			if (dir > 0) w.y = -w.y;
			float2* a = s + line * LS;
			const float2 u = a[k0], v = a[k1];
			const float2 t = make_float2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
			a[k0] = make_float2(u.x + t.x, u.y + t.y);
			a[k1] = make_float2(u.x - t.x, u.y - t.y);
		}
		__syncthreads();
	}
}

template <int N>
__device__ __forceinline__ int bitrev(int k) {
	return (int)(__brev((unsigned)k) >> (32 - ilog2c(N)));
}

// A launch covers nitem images.  WFS mode: image i is subaperture i / nw of
// wfs[i % nw] (the order of the 32-point launches).  Uplink mode: image i is
// the LLT pupil of wfs[i] (opd = LLT OPD, amp = LLT amplitude), and pass 4
// stores its OTF, transposed, into wfs[i].lotfT instead of applying it.
struct GenParams {
	int nitem, nw, nopd, pad;
	int uplink;
	float scale;                 // factor on |.|^2: 1 for WFS images, 1/N^2 for LLT pupils
	float twoinvwvl;
	float2* buf;                 // nitem * N * N scratch, row-major per image
	const float2* tw;            // N/2 twiddles exp(-2 pi i k / N)
	const WfsDev* wfs;
	const float2* etfT1;         // nsa * N^2 transposed, or null
	const float2* etfT2;
	float etfwt1, etfwt2;
	const float* nominalT;       // N^2 (or nsa * N^2) transposed, or null
	int nominal_per_sa;
};

// One pass over one tile (blockIdx.y) of one image (blockIdx.x).
template <int N, int PASS>
__global__ void __launch_bounds__(GEN_THREADS) gen_pass_kernel(GenParams G) {
	constexpr int LS = N + 1, GEN_LINES = gen_lines(N);
	constexpr bool ROWS = PASS == GEN_FIELD_ROWS || PASS == GEN_OTF_ROWS || PASS == GEN_INV_ROWS;
	extern __shared__ float2 gen_s[];
	float2* tw = gen_s + GEN_LINES * LS;  // N/2 twiddles
	const int i = blockIdx.x;
	const int isa = G.uplink ? 0 : i / G.nw;
	const WfsDev& W = G.wfs[G.uplink ? i : i % G.nw];
	float2* im = G.buf + (size_t)i * N * N;
	const int tid = threadIdx.x;
	for (int k = tid; k < N / 2; k += GEN_THREADS) tw[k] = G.tw[k];
	int l0 = blockIdx.y * GEN_LINES, nl = GEN_LINES;  // first line and lines of the tile
	if (PASS == GEN_FIELD_ROWS) {
		nl = min(GEN_LINES, G.nopd - l0);
		l0 += G.pad;
	}
	// ---- load (bit-reversed along the line)
	for (int idx = tid; idx < GEN_LINES * N; idx += GEN_THREADS) {
		int line, k;
		if (ROWS) {
			line = idx / N;
			k = idx - line * N;
		} else {
			k = idx / GEN_LINES;
			line = idx - k * GEN_LINES;
		}
		float2 v = make_float2(0.f, 0.f);
		if (line < nl) {
			if (PASS == GEN_FIELD_ROWS) {
				const int x = k - G.pad, y = l0 + line - G.pad;
				if (x >= 0 && x < G.nopd) {
					const size_t e = (size_t)isa * G.nopd * G.nopd + (size_t)y * G.nopd + x;
					const float o = __ldg(W.opd + e), a = __ldg(W.amp + e);
					float sn, cs;
					sincospif(G.twoinvwvl * o, &sn, &cs);
					v = make_float2(a * cs, a * sn);
				}
			} else if (ROWS) {
				v = im[(size_t)(l0 + line) * N + k];
			} else if (PASS != GEN_PSF_COLS || (k >= G.pad && k < G.pad + G.nopd)) {
				v = im[(size_t)k * N + l0 + line];  // rows outside the pupil are zero before pass 2
			}
		}
		gen_s[line * LS + bitrev<N>(k)] = v;
	}
	__syncthreads();
	fft_lines<N>(gen_s, tw, PASS >= GEN_INV_ROWS ? 1 : -1);
	// ---- element-wise step of the chain
	if (PASS == GEN_PSF_COLS) {
		for (int idx = tid; idx < GEN_LINES * N; idx += GEN_THREADS) {
			const float2 v = gen_s[(idx / N) * LS + idx % N];
			gen_s[(idx / N) * LS + idx % N] = make_float2((v.x * v.x + v.y * v.y) * G.scale, 0.f);
		}
		__syncthreads();
	}
	if (PASS == GEN_OTF_COLS) {
		// line = fx - l0, element fy; transfer functions are [fy + N fx]: fy fastest
		for (int idx = tid; idx < GEN_LINES * N; idx += GEN_THREADS) {
			const int line = idx / N, fy = idx - line * N;
			const size_t t = (size_t)fy + (size_t)N * (l0 + line);
			float2 v = gen_s[line * LS + fy];
			if (G.uplink) {
				const_cast<float2*>(W.lotfT)[t] = v;  // the uplink OTF this launch produces
				continue;
			}
			if (W.lotfT) v = cmulc(v, __ldg(W.lotfT + t));
			if (G.etfT1) {
				float2 e = __ldg(G.etfT1 + (size_t)isa * N * N + t);
				if (G.etfT2) {
					const float2 e2 = __ldg(G.etfT2 + (size_t)isa * N * N + t);
					e = make_float2(e.x * G.etfwt1 + e2.x * G.etfwt2, e.y * G.etfwt1 + e2.y * G.etfwt2);
				}
				v = cmul(v, e);
			} else if (G.nominalT) {
				const float d = __ldg(G.nominalT + (G.nominal_per_sa ? (size_t)isa * N * N : 0) + t);
				v = make_float2(v.x * d, v.y * d);
			}
			gen_s[line * LS + fy] = v;
		}
		__syncthreads();
		if (G.uplink) return;
	}
	if (PASS == GEN_INV_COLS) {
		for (int idx = tid; idx < GEN_LINES * N; idx += GEN_THREADS) {
			const int line = idx / N, k = idx - line * N;
			gen_s[line * LS + k].y = 0.f;  // real part only
		}
		__syncthreads();
	}
	// ---- store (natural order)
	for (int idx = tid; idx < GEN_LINES * N; idx += GEN_THREADS) {
		int line, k;
		if (ROWS) {
			line = idx / N;
			k = idx - line * N;
		} else {
			k = idx / GEN_LINES;
			line = idx - k * GEN_LINES;
		}
		if (line < nl) {
			if (ROWS) im[(size_t)(l0 + line) * N + k] = gen_s[line * LS + k];
			else im[(size_t)k * N + l0 + line] = gen_s[line * LS + k];
		}
	}
}

// Pixels, noise and gradients of generic-size images: one warp per work item
// (item = isa * nw + k as in the imaging launch), image item of buf (n2 = N^2
// elements each), real part.
template <int NPQ>
__global__ void gen_pixels_kernel(PowfsDev P, const WfsDev* __restrict__ wfs, int nw, int nitem,
	const float2* __restrict__ buf, int n2) {
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int item = blockIdx.x * (blockDim.x >> 5) + warp;
	if (item >= nitem) return;
	const int isa = item / nw;
	const WfsDev& W = wfs[item % nw];
	const float2* im = buf + (size_t)item * n2;
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
				if (id >= 0) v = fmaf(__ldg(swt + 4 * p + c), im[id].x, v);
			}
			v *= W.alpha;
		}
		pix[q] = v;
	}
	if (W.noisy) {
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) {
				PixelRng rng(W.seed, (uint32_t)(isa * npix + p), W.wfs_id, (uint32_t)P.isim);
				pix[q] = poisson_draw(rng, pix[q] + P.bkgrnd) + P.rne * rng.normal() - P.bkgrndc;
			}
		}
	}
	if (W.ints) {
#pragma unroll
		for (int q = 0; q < NPQ; q++) {
			const int p = lane + 32 * q;
			if (p < npix) W.ints[(size_t)isa * npix + p] = pix[q];
		}
	}
	if (W.grad)
		grad_from_pixels<NPQ>(pix, npix, P.pixpsax, P.pixpsay, P, W.mtche + (size_t)isa * 2 * npix, W.i0sum, isa, lane,
			W.grad, P.nsa);
}

}  // namespace shwfs
