// Imaging stages (b)-(e) for the larger FFT sizes, n_f = n_w = N in {64, 128,
// 256} (the NGS and tip-tilt sensors of an uneven batch, large-sampling LGS):
// a chain of batched 1-D FFT passes over a per-powfs scratch image in global
// memory (L2-resident for the small batches), each pass a kernel that moves
// tiles of 16 rows or 16 columns of an image through shared memory, with the
// element-wise step of the chain fused in:
//
//   pass 1  columns x in [pad, pad+n_o): field E = amp exp(i 2 pi opd / lambda), FFT along y
//   pass 2  rows ky:                     FFT along x (columns outside the pupil are zero),
//                                        |.|^2 * scale, FFT along x (the PSF's transform)
//   pass 3  columns fx:                  FFT along ky (the OTF), x conj(uplink OTF) x ETF / DTF
//                                        nominal, inverse FFT along fy
//   pass 4  rows y:                      inverse FFT along fx, real part
//   pixels  a thread per pixel:          bilinear pixel map, noise, CoG / matched filter
//
// The two-dimensional transforms are separable, so each pass takes its lines
// through two of them where the chain allows (the PSF's rows right after the
// field's, the inverse's columns right after the OTF's): four passes over the
// image instead of six, with the same transforms and element-wise steps
// as maos/wfsints.c:233-286 (cembed_wvf with pad (n_w - n_o)/2, cfft2 with
// FFTW's sign and no normalisation, cabs2toreal, ccwmc with the uplink OTF,
// apply_dtf_etf, cfft2 inverse, dspmulcreal).  For the LLT pupil, passes 1-3
// up to the OTF give the uplink OTF (maos/wfsints.c:149-199).
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

enum GenPass { GEN_FIELD_COLS = 1, GEN_PSF_ROWS, GEN_OTF_COLS, GEN_INV_ROWS };
constexpr int GEN_NPASS = 4;

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// Radix-2 decimation-in-time butterfly: (u, v) -> (u + w v, u - w v).
__device__ __forceinline__ void gen_bfly(float2& u, float2& v, float2 w) {
	const float2 t = make_float2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
	v = make_float2(u.x - t.x, u.y - t.y);
	u = make_float2(u.x + t.x, u.y + t.y);
}

// In-place FFT of gen_lines(N) lines of N points in shared memory, line stride
// N + 1 (bank-conflict free for column tiles), input in bit-reversed order.
// tw[k] = exp(-2 pi i k / N), k < N/2; dir -1 forward, +1 inverse.  The
// log2 N radix-2 stages run two at a time: a thread takes the four points
// k0 + {0, h, 2h, 3h} (h = 2^st) and applies stage st's butterflies (k0, k0+h)
// and (k0+2h, k0+3h), then stage st+1's (k0, k0+2h) and (k0+h, k0+3h), with
// those stages' twiddles -- every point sees the operations of the stage-by-
// stage transform in the same order, with half its barriers and shared-memory
// round trips (an odd log2 N starts with one radix-2 stage).
template <int N, int NT = GEN_THREADS>
__device__ __forceinline__ void fft_lines(float2* s, const float2* __restrict__ tw, int dir) {
	constexpr int LOGN = ilog2c(N), LS = N + 1, NB = gen_lines(N) * N / 2, NQ = gen_lines(N) * N / 4;
	int st = 0;
	if (LOGN & 1) {  // stage 0: half = 1, twiddle tw[0]
		float2 w0 = tw[0];
		if (dir > 0) w0.y = -w0.y;
		for (int b = threadIdx.x; b < NB; b += NT) {
			const int line = b / (N / 2), j = b - line * (N / 2);
			float2* a = s + line * LS + 2 * j;
			float2 u = a[0], v = a[1];
			gen_bfly(u, v, w0);
			a[0] = u;
			a[1] = v;
		}
		__syncthreads();
		st = 1;
	}
#pragma unroll 1
	for (; st < LOGN; st += 2) {
		const int h = 1 << st;
		for (int b = threadIdx.x; b < NQ; b += NT) {
			const int line = b / (N / 4), j = b - line * (N / 4);
			const int grp = j >> st, pos = j & (h - 1);
			float2* a = s + line * LS + grp * 4 * h + pos;
			float2 w1 = tw[pos << (LOGN - 1 - st)];
			float2 w2 = tw[pos << (LOGN - 2 - st)], w3 = tw[(pos + h) << (LOGN - 2 - st)];
			if (dir > 0) {
				w1.y = -w1.y;
				w2.y = -w2.y;
				w3.y = -w3.y;
			}
			float2 x0 = a[0], x1 = a[h], x2 = a[2 * h], x3 = a[3 * h];
			gen_bfly(x0, x1, w1);  // stage st
			gen_bfly(x2, x3, w1);
			gen_bfly(x0, x2, w2);  // stage st + 1
			gen_bfly(x1, x3, w3);
			a[0] = x0;
			a[h] = x1;
			a[2 * h] = x2;
			a[3 * h] = x3;
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
// the LLT pupil of wfs[i] (opd = LLT OPD, amp = LLT amplitude), and pass 3
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

// Shared memory of one pass tile: the lines (stride N + 1) and N/2 twiddles.
__host__ __device__ constexpr int gen_tile_smem(int n) { return (gen_lines(n) * (n + 1) + n / 2) * (int)sizeof(float2); }

// Reads of the scratch image: through L1, or from L2 only (L2ONLY) where other
// blocks of the same launch wrote it (L1 is not coherent between SMs).
template <bool L2ONLY>
__device__ __forceinline__ float2 gen_ld(const float2* p) {
	if constexpr (L2ONLY) return __ldcg(p);
	else return *p;
}

// Element-wise step f(value, line, k) over a tile's lines in natural order,
// the results left in bit-reversed order along each line for the line's next
// transform (a pass that transforms its lines twice).
template <int N, int NT, typename F>
__device__ __forceinline__ void gen_permute(float2* s, F f) {
	constexpr int LS = N + 1, NE = gen_lines(N) * N / NT;
	static_assert(gen_lines(N) * N % NT == 0, "tile elements per thread");
	float2 v[NE];
#pragma unroll
	for (int e = 0; e < NE; e++) {
		const int idx = threadIdx.x + e * NT, line = idx / N, k = idx - line * N;
		v[e] = f(s[line * LS + k], line, k);
	}
	__syncthreads();
#pragma unroll
	for (int e = 0; e < NE; e++) {
		const int idx = threadIdx.x + e * NT, line = idx / N, k = idx - line * N;
		s[line * LS + bitrev<N>(k)] = v[e];
	}
	__syncthreads();
}

// One pass over tile `tile` of image i by a block of NT threads; gen_s is the
// tile's shared memory (gen_tile_smem(N) bytes).
template <int N, int PASS, int NT, bool L2ONLY>
__device__ __forceinline__ void gen_pass_tile(const GenParams& G, int i, int tile, float2* gen_s) {
	constexpr int LS = N + 1, GEN_LINES = gen_lines(N);
	constexpr bool ROWS = PASS == GEN_PSF_ROWS || PASS == GEN_INV_ROWS;
	float2* tw = gen_s + GEN_LINES * LS;  // N/2 twiddles
	const int isa = G.uplink ? 0 : i / G.nw;
	const WfsDev& W = G.wfs[G.uplink ? i : i % G.nw];
	float2* im = G.buf + (size_t)i * N * N;
	const int tid = threadIdx.x;
	for (int k = tid; k < N / 2; k += NT) tw[k] = G.tw[k];
	int l0 = tile * GEN_LINES, nl = GEN_LINES;  // first line and lines of the tile
	if (PASS == GEN_FIELD_COLS) {  // only the pupil's columns
		nl = min(GEN_LINES, G.nopd - l0);
		l0 += G.pad;
	}
	// ---- load (bit-reversed along the line)
	for (int idx = tid; idx < GEN_LINES * N; idx += NT) {
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
			if (PASS == GEN_FIELD_COLS) {
				const int x = l0 + line - G.pad, y = k - G.pad;
				if (y >= 0 && y < G.nopd) {
					const size_t e = (size_t)isa * G.nopd * G.nopd + (size_t)y * G.nopd + x;
					const float o = __ldg(W.opd + e), a = __ldg(W.amp + e);
					float sn, cs;
					sincospif(G.twoinvwvl * o, &sn, &cs);
					v = make_float2(a * cs, a * sn);
				}
			} else if (!ROWS) {
				v = gen_ld<L2ONLY>(im + (size_t)k * N + l0 + line);
			} else if (PASS != GEN_PSF_ROWS || (k >= G.pad && k < G.pad + G.nopd)) {
				v = gen_ld<L2ONLY>(im + (size_t)(l0 + line) * N + k);  // columns outside the pupil are zero
			}
		}
		gen_s[line * LS + bitrev<N>(k)] = v;
	}
	__syncthreads();
	fft_lines<N, NT>(gen_s, tw, PASS == GEN_INV_ROWS ? 1 : -1);
	// ---- element-wise steps of the chain, and a pass's second transform
	if (PASS == GEN_PSF_ROWS) {
		// |.|^2 * scale: the PSF row, then its own transform along x (the OTF's)
		gen_permute<N, NT>(gen_s, [&](float2 v, int, int) { return make_float2((v.x * v.x + v.y * v.y) * G.scale, 0.f); });
		fft_lines<N, NT>(gen_s, tw, -1);
	}
	if (PASS == GEN_OTF_COLS) {
		// line = fx - l0, element fy: the OTF; transfer functions are [fy + N fx], fy fastest
		if (G.uplink) {
			for (int idx = tid; idx < GEN_LINES * N; idx += NT) {
				const int line = idx / N, fy = idx - line * N;
				const_cast<float2*>(W.lotfT)[(size_t)fy + (size_t)N * (l0 + line)] = gen_s[line * LS + fy];  // the uplink OTF
			}
			return;
		}
		gen_permute<N, NT>(gen_s, [&](float2 v, int line, int fy) {
			const size_t t = (size_t)fy + (size_t)N * (l0 + line);
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
			return v;
		});
		fft_lines<N, NT>(gen_s, tw, 1);  // the inverse along fy
	}
	// ---- store (natural order; the last pass keeps the real part)
	for (int idx = tid; idx < GEN_LINES * N; idx += NT) {
		int line, k;
		if (ROWS) {
			line = idx / N;
			k = idx - line * N;
		} else {
			k = idx / GEN_LINES;
			line = idx - k * GEN_LINES;
		}
		if (line < nl) {
			float2 v = gen_s[line * LS + k];
			if (PASS == GEN_INV_ROWS) v.y = 0.f;
			if (ROWS) im[(size_t)(l0 + line) * N + k] = v;
			else im[(size_t)k * N + l0 + line] = v;
		}
	}
}

// One pass over one tile (blockIdx.y) of one image (blockIdx.x).
template <int N, int PASS>
__global__ void __launch_bounds__(GEN_THREADS) gen_pass_kernel(GenParams G) {
	extern __shared__ float2 gen_s[];
	gen_pass_tile<N, PASS, GEN_THREADS, false>(G, blockIdx.x, blockIdx.y, gen_s);
}

// Pixels, noise and gradients of generic-size images: one warp per work item
// (item = isa * nw + k as in the imaging launch), image item of buf (n2 = N^2
// elements each), real part.
template <int NPQ, bool L2ONLY>
__device__ __forceinline__ void gen_pixels_item(const PowfsDev& P, const WfsDev* __restrict__ wfs, int nw, int item,
	const float2* __restrict__ buf, int n2, int lane) {
	const int isa = item / nw;
	const WfsDev& W = wfs[item % nw];
	const float2* im = buf + (size_t)item * n2;
	const int npix = P.npix;
	// a pixel's 4 map entries are one 16-byte row (cudaMalloc'd, 4 entries per pixel)
	const int4* sidx = reinterpret_cast<const int4*>(P.simap_idx) + (P.simap_per_sa ? (size_t)isa * npix : 0);
	const float4* swt = reinterpret_cast<const float4*>(P.simap_wt) + (P.simap_per_sa ? (size_t)isa * npix : 0);
	// Few warps run these images, so every load latency is exposed: the map
	// rows, then the image taps, are each issued as one independent wave.  A
	// missing tap (index < 0) reads as 0, and fmaf(w, 0, v) = v, so the sums
	// equal those that skip it.
	float x[NPQ][4];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		const int4 id = p < npix ? __ldg(sidx + p) : make_int4(-1, -1, -1, -1);
		x[q][0] = id.x >= 0 ? gen_ld<L2ONLY>(im + id.x).x : 0.f;
		x[q][1] = id.y >= 0 ? gen_ld<L2ONLY>(im + id.y).x : 0.f;
		x[q][2] = id.z >= 0 ? gen_ld<L2ONLY>(im + id.z).x : 0.f;
		x[q][3] = id.w >= 0 ? gen_ld<L2ONLY>(im + id.w).x : 0.f;
	}
	float pix[NPQ];
#pragma unroll
	for (int q = 0; q < NPQ; q++) {
		const int p = lane + 32 * q;
		float v = 0.f;
		if (p < npix) {
			const float4 w = __ldg(swt + p);
			v = fmaf(w.x, x[q][0], v);
			v = fmaf(w.y, x[q][1], v);
			v = fmaf(w.z, x[q][2], v);
			v = fmaf(w.w, x[q][3], v);
			v *= W.alpha;
			if (P.accum) v += W.ints[(size_t)isa * npix + p];  // dtrat > 1: the frames so far
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
// The same step with one block per image (blockIdx.x = item), a thread per
// pixel (npix rounded up to whole warps): the launches of these sizes often
// hold a few images, where a warp walking 8 pixels' noise draws in turn set
// their latency.  The
// image's first warp then forms the gradients from the pixels in shared
// memory, in gen_pixels_item's lane order (pixel p = lane + 32 q), so
// intensities, noise and gradients equal those of gen_pixels_item.
constexpr int GEN_PIX_THREADS = 256;  // the largest pixel count of these sizes
__global__ void __launch_bounds__(GEN_PIX_THREADS) gen_pixels_block_kernel(PowfsDev P,
	const WfsDev* __restrict__ wfs, int nw, const float2* __restrict__ buf, int n2) {
	__shared__ float spix[GEN_PIX_THREADS];
	const int item = blockIdx.x, p = threadIdx.x;
	const int isa = item / nw;
	const WfsDev& W = wfs[item % nw];
	const int npix = P.npix;
	float v = 0.f;
	if (p < npix) {
		const float2* im = buf + (size_t)item * n2;
		const size_t m = (P.simap_per_sa ? (size_t)isa * npix : 0) + p;
		const int4 id = __ldg(reinterpret_cast<const int4*>(P.simap_idx) + m);
		const float4 w = __ldg(reinterpret_cast<const float4*>(P.simap_wt) + m);
		v = fmaf(w.x, id.x >= 0 ? im[id.x].x : 0.f, v);
		v = fmaf(w.y, id.y >= 0 ? im[id.y].x : 0.f, v);
		v = fmaf(w.z, id.z >= 0 ? im[id.z].x : 0.f, v);
		v = fmaf(w.w, id.w >= 0 ? im[id.w].x : 0.f, v);
		v *= W.alpha;
		if (P.accum) v += W.ints[(size_t)isa * npix + p];  // dtrat > 1: the frames so far
		if (W.noisy) {
			PixelRng rng(W.seed, (uint32_t)(isa * npix + p), W.wfs_id, (uint32_t)P.isim);
			v = poisson_draw(rng, v + P.bkgrnd) + P.rne * rng.normal() - P.bkgrndc;
		}
		if (W.ints) W.ints[(size_t)isa * npix + p] = v;
	}
	spix[p] = v;
	__syncthreads();
	if (p < 32 && W.grad) {
		float pix[GEN_PIX_THREADS / 32];
#pragma unroll
		for (int q = 0; q < GEN_PIX_THREADS / 32; q++) pix[q] = p + 32 * q < npix ? spix[p + 32 * q] : 0.f;
		grad_from_pixels<GEN_PIX_THREADS / 32>(pix, npix, P.pixpsax, P.pixpsay, P, W.mtche + (size_t)isa * 2 * npix,
			W.i0sum, isa, p, W.grad, P.nsa);
	}
}

// ---------------------------------------------------------------------------
// n_f = n_w = 64 fused per image: one block of 256 threads holds the 64x64
// image in shared memory; every 64-point line transform is 8 x 8: n = 8 n1 +
// n2, k = k1 + 8 k2, X[k] = sum_n2 w64^(n2 k1) w8^(n2 k2) sum_n1 x[n] w8^(n1 k1),
// with the 8-point transforms in registers, so each line costs two passes
// through shared memory.  Form F takes the line in natural order and leaves
// X[k] at the digit-reversed position r(k) = 8 (k mod 8) + k / 8; form G takes
// the line in digit-reversed order and leaves it natural.  The chain uses F
// for the field and the inverse transforms and G for the PSF -> OTF transform,
// so the OTF is in natural order where the transfer functions multiply it, and
// the final image sits at digit-reversed rows and columns.
// ---------------------------------------------------------------------------
constexpr int N64_LS = 65;  // line stride of the shared image (float2): row, column and
                            // transfer-function accesses all at the 2-wavefront minimum

__device__ __forceinline__ int digrev8(int k) { return ((k & 7) << 3) | (k >> 3); }

// 8-point DFT in registers, natural order in and out; dir -1 forward, +1 inverse
__device__ __forceinline__ void dft8(float2 (&a)[8], float dir) {
	const float h = 0.70710678118654752f;
	// radix-2 stage on pairs (j, j+4)
	float2 b[8];
#pragma unroll
	for (int j = 0; j < 4; j++) {
		b[j] = make_float2(a[j].x + a[j + 4].x, a[j].y + a[j + 4].y);
		b[j + 4] = make_float2(a[j].x - a[j + 4].x, a[j].y - a[j + 4].y);
	}
	// twiddles w8^j on b[4..7]: w8 = exp(dir i pi/4)
	{
		float2 t = b[5];
		b[5] = make_float2(h * (t.x - dir * t.y), h * (t.y + dir * t.x));
		t = b[6];
		b[6] = make_float2(-dir * t.y, dir * t.x);
		t = b[7];
		b[7] = make_float2(h * (-t.x - dir * t.y), h * (-t.y + dir * t.x));
	}
	// two 4-point DFTs: (b0..b3) -> even outputs, (b4..b7) -> odd outputs
#pragma unroll
	for (int g = 0; g < 2; g++) {
		const float2 c0 = b[4 * g], c1 = b[4 * g + 1], c2 = b[4 * g + 2], c3 = b[4 * g + 3];
		const float2 s0 = make_float2(c0.x + c2.x, c0.y + c2.y), d0 = make_float2(c0.x - c2.x, c0.y - c2.y);
		const float2 s1 = make_float2(c1.x + c3.x, c1.y + c3.y), d1 = make_float2(c1.x - c3.x, c1.y - c3.y);
		const float2 d1r = make_float2(-dir * d1.y, dir * d1.x);  // d1 * (dir i)
		a[g] = make_float2(s0.x + s1.x, s0.y + s1.y);                // X[0] / X[1]
		a[g + 2] = make_float2(d0.x + d1r.x, d0.y + d1r.y);          // X[2] / X[3]
		a[g + 4] = make_float2(s0.x - s1.x, s0.y - s1.y);            // X[4] / X[5]
		a[g + 6] = make_float2(d0.x - d1r.x, d0.y - d1r.y);          // X[6] / X[7]
	}
}

// One 64-point transform of NLINES lines (nlines when NLINES is 0) of the
// 64 x N64_LS shared image: rows (line L at s + (line0 + L) * N64_LS, element
// j at + j) or columns (COLS: line L at s + line0 + L, element j at + j *
// N64_LS), in form F (DIGREV_IN false) or G (true), DIR -1 forward, +1
// inverse.  In form F the input elements outside [lo, hi) are taken as zero
// and not read (a zero-padded field needs no zero fill).  Called by all
// N64_THREADS threads of the block.
// tw[k] = exp(-2 pi i k / 64).
constexpr int N64_THREADS = 256;
template <bool DIGREV_IN, bool COLS, int NLINES, int DIR>
__device__ __forceinline__ void fft64_lines(float2* s, int line0, const float2* __restrict__ tw, int nlines = NLINES,
	int lo = 0, int hi = 64) {
	constexpr int ls = COLS ? 1 : N64_LS, es = COLS ? N64_LS : 1;
	constexpr float dir = (float)DIR;
	const unsigned nl = NLINES > 0 ? (unsigned)NLINES : (unsigned)nlines;
#pragma unroll
	for (int step = 0; step < 2; step++) {
		// F: step 0 gathers 8 i + t and twiddles, step 1 gathers 8 t + i.
		// G: step 0 gathers 8 t + i and twiddles, step 1 gathers 8 i + t.
		const bool strided = (step == 0) != DIGREV_IN;
		const unsigned ntask = nl * 8;
		// consecutive threads take consecutive lines for column lines, and for
		// the gather of 8 consecutive elements of row lines (rows are N64_LS
		// apart: conflict-free), consecutive tasks for the strided gather of row
		// lines (consecutive elements)
		const bool lines_fast = COLS || !strided;
		for (unsigned task = threadIdx.x; task < ntask; task += N64_THREADS) {
			unsigned L, t;
			if (lines_fast) {
				L = task % nl;
				t = task / nl;
			} else {
				L = task >> 3;
				t = task & 7;
			}
			float2* line = s + (line0 + L) * ls;
			float2 a[8];
#pragma unroll
			for (int i = 0; i < 8; i++) {
				const int j = strided ? 8 * i + (int)t : 8 * (int)t + i;
				if (!DIGREV_IN && step == 0)
					a[i] = (j >= lo && j < hi) ? line[j * es] : make_float2(0.f, 0.f);
				else
					a[i] = line[j * es];
			}
			dft8(a, dir);
			if (step == 0) {
#pragma unroll
				for (int i = 1; i < 8; i++) {
					float2 w = tw[(t * i) & 63u];
					w.y *= -dir;  // tw holds exp(-...); dir -1 keeps it, +1 conjugates
					const float2 v = a[i];
					a[i] = make_float2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
				}
			}
#pragma unroll
			for (int i = 0; i < 8; i++) line[(strided ? 8 * i + (int)t : 8 * (int)t + i) * es] = a[i];
		}
		__syncthreads();
	}
}

// (b)-(e) fused for n_f = n_w = 64: one block per work item (item = isa * nw +
// k as in the other imaging launches).  Dynamic shared memory
// N64_SMEM_BYTES.  tw64[k] = exp(-2 pi i k / 64), k < 64.
constexpr int N64_SMEM_BYTES = (64 * N64_LS + 64) * 8 + 256 * 4;
// NOPD > 0 fixes the pupil size at compile time (nopd is then ignored).
template <int NOPD>
__global__ void __launch_bounds__(N64_THREADS, 6) ints_n64_kernel(PowfsDev P, const WfsDev* __restrict__ wfs, int nw,
	int nitem, int nopd_rt, float twoinvwvl, const float2* __restrict__ tw64) {
	const int nopd = NOPD > 0 ? NOPD : nopd_rt;
	extern __shared__ float2 n64_s[];
	float2* img = n64_s;
	float2* tw = n64_s + 64 * N64_LS;
	float* spix = reinterpret_cast<float*>(tw + 64);
	const int item = blockIdx.x, tid = threadIdx.x;
	if (item >= nitem) return;
	const int isa = item / nw;
	const WfsDev& W = wfs[item % nw];
	const int pad = (64 - nopd) / 2, no2 = nopd * nopd;
	if (tid < 64) tw[tid] = tw64[tid];
	// (b) field, zero-padded (cembed_wvf, maos/wfsints.c:233): only the pupil
	// square is written; the first transforms read nothing outside it
	for (int idx = tid; idx < no2; idx += N64_THREADS) {
		const int y = idx / nopd, x = idx - y * nopd;
		const float o = __ldg(W.opd + (size_t)isa * no2 + idx), a = __ldg(W.amp + (size_t)isa * no2 + idx);
		float sn, cs;
		sincospif(twoinvwvl * o, &sn, &cs);
		img[(y + pad) * N64_LS + x + pad] = make_float2(a * cs, a * sn);
	}
	__syncthreads();
	// (c) PSF: forward along x on the pupil rows, along y
	fft64_lines<false, false, NOPD, -1>(img, pad, tw, nopd, pad, pad + nopd);
	fft64_lines<false, true, 64, -1>(img, 0, tw, 64, pad, pad + nopd);
	// |.|^2, two real PSF rows per complex row: row r <- (PSF row r) + i (PSF row r + 32)
	for (int idx = tid; idx < 32 * 64; idx += N64_THREADS) {
		float2* v = img + (idx >> 6) * N64_LS + (idx & 63);
		const float2 a = v[0], b = v[32 * N64_LS];
		v[0] = make_float2(a.x * a.x + a.y * a.y, b.x * b.x + b.y * b.y);
	}
	__syncthreads();
	// OTF, half spectrum kx = 0..32 (the PSF is real, so OTF(-k) = conj OTF(k)):
	// forward along kx on the 32 packed rows (digit-reversed inputs)
	fft64_lines<true, false, 32, -1>(img, 0, tw);
	// unpack the pairs: row r's spectrum Z = H_r + i H_{r+32}, H_r(kx) = (Z(kx) +
	// conj Z(-kx)) / 2, H_{r+32}(kx) = (Z(kx) - conj Z(-kx)) / 2i.  H(0) and
	// H(32) are real, so column 0 carries H(0) + i H(32) and column 32 is free.
	for (int idx = tid; idx < 32 * 32; idx += N64_THREADS) {
		const int r = idx >> 5, kx = idx & 31;
		float2* row = img + r * N64_LS;
		const float2 z = row[kx], zm = row[kx ? 64 - kx : 32];
		if (kx) {
			row[kx] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
			row[32 * N64_LS + kx] = make_float2(0.5f * (z.y + zm.y), 0.5f * (zm.x - z.x));
		} else {
			row[0] = make_float2(z.x, zm.x);
			row[32 * N64_LS] = make_float2(z.y, zm.y);
		}
	}
	__syncthreads();
	// forward along ky on columns 0..31 (digit-reversed inputs): natural OTF
	fft64_lines<true, true, 32, -1>(img, 0, tw);
	// x conj(uplink OTF) x ETF / nominal; transfer functions are [fy + 64 fx].
	// Column 0 holds
	// Y = O(.,0) + i O(.,32) with O(.,0), O(.,32) the transforms of real
	// columns; the products for kx = 0 and 32 go to column 32 as X(.,0) + i X(.,32).
	{
		const float2* e1 = P.etfT1 ? P.etfT1 + (size_t)isa * 4096 : nullptr;
		const float2* e2 = P.etfT2 ? P.etfT2 + (size_t)isa * 4096 : nullptr;
		const float* nm = P.nominalT ? P.nominalT + (P.nominal_per_sa ? (size_t)isa * 4096 : 0) : nullptr;
		auto tf = [&](int t) -> float2 {
			float2 o = make_float2(1.f, 0.f);
			if (W.lotfT) {
				const float2 l = __ldg(W.lotfT + t);
				o = make_float2(l.x, -l.y);
			}
			if (e1) {
				float2 e = __ldg(e1 + t);
				if (e2) {
					const float2 f = __ldg(e2 + t);
					e = make_float2(e.x * P.etfwt1 + f.x * P.etfwt2, e.y * P.etfwt1 + f.y * P.etfwt2);
				}
				o = cmul(o, e);
			} else if (nm) {
				const float d = __ldg(nm + t);
				o = make_float2(o.x * d, o.y * d);
			}
			return o;
		};
		// The transfer functions are transforms of real kernels (uplink PSF,
		// elongated spot, pixel response), Hermitian to rounding, so each
		// half-spectrum element takes TF(t) itself: the image is then the real
		// part of the full inverse up to rounding.
		for (int t = tid; t < 64 * 32; t += N64_THREADS) {
			const int fy = t & 63, fx = t >> 6, my = (64 - fy) & 63;
			if (fx) {
				float2* v = img + fy * N64_LS + fx;
				*v = cmul(*v, tf(t));
			} else {
				const float2 y = img[fy * N64_LS], ym = img[my * N64_LS];
				const float2 o0 = make_float2(0.5f * (y.x + ym.x), 0.5f * (y.y - ym.y));
				const float2 o32 = make_float2(0.5f * (y.y + ym.y), 0.5f * (ym.x - y.x));
				const float2 x0 = cmul(o0, tf(fy)), x32 = cmul(o32, tf(fy + 64 * 32));
				img[fy * N64_LS + 32] = make_float2(x0.x - x32.y, x0.y + x32.x);
			}
		}
	}
	__syncthreads();
	// inverse along fy on columns 1..32: G(y, kx) at digit-reversed rows, column
	// 32 holding G(., 0) + i G(., 32) (both real)
	fft64_lines<false, true, 32, 1>(img, 1, tw);
	// two real image rows per complex row: row r <- a + i b over the full kx
	// range, a and b the Hermitian extensions of rows r and r + 32
	for (int idx = tid; idx < 32 * 32; idx += N64_THREADS) {
		const int r = idx >> 5, kx = idx & 31;
		float2* row = img + r * N64_LS;
		if (kx) {
			const float2 a = row[kx], b = row[32 * N64_LS + kx];
			row[kx] = make_float2(a.x - b.y, a.y + b.x);
			row[64 - kx] = make_float2(a.x + b.y, b.x - a.y);
		} else {
			const float2 a = row[32], b = row[32 * N64_LS + 32];
			row[0] = make_float2(a.x, b.x);
			row[32] = make_float2(a.y, b.y);
		}
	}
	__syncthreads();
	// inverse along fx on the 32 packed rows: image row s (digit-reversed) is the
	// real part of row s for s < 32, the imaginary part of row s - 32 otherwise
	fft64_lines<false, false, 32, 1>(img, 0, tw);
	// (d) pixels (bilinear map) and noise, one thread per pixel
	const int npix = P.npix;
	const int* sidx = P.simap_idx + (P.simap_per_sa ? (size_t)isa * npix * 4 : 0);
	const float* swt = P.simap_wt + (P.simap_per_sa ? (size_t)isa * npix * 4 : 0);
	for (int p = tid; p < npix; p += N64_THREADS) {
		float v = 0.f;
#pragma unroll
		for (int c = 0; c < 4; c++) {
			const int id = __ldg(sidx + 4 * p + c);
			if (id >= 0) {
				const int sr = digrev8(id >> 6);
				const float2 q = img[(sr & 31) * N64_LS + digrev8(id & 63)];
				v = fmaf(__ldg(swt + 4 * p + c), sr < 32 ? q.x : q.y, v);
			}
		}
		v *= W.alpha;
		if (P.accum) v += W.ints[(size_t)isa * npix + p];  // dtrat > 1: the frames so far
		if (W.noisy) {
			PixelRng rng(W.seed, (uint32_t)(isa * npix + p), W.wfs_id, (uint32_t)P.isim);
			v = poisson_draw(rng, v + P.bkgrnd) + P.rne * rng.normal() - P.bkgrndc;
		}
		if (W.ints) W.ints[(size_t)isa * npix + p] = v;
		spix[p] = v;
	}
	__syncthreads();
	// (e) gradients
	if (tid < 32 && W.grad) {
		float pix[8];
#pragma unroll
		for (int q = 0; q < 8; q++) {
			const int p = tid + 32 * q;
			pix[q] = p < npix ? spix[p] : 0.f;
		}
		grad_from_pixels<8>(pix, npix, P.pixpsax, P.pixpsay, P, W.mtche + (size_t)isa * 2 * npix, W.i0sum, isa, tid,
			W.grad, P.nsa);
	}
}

}  // namespace shwfs
