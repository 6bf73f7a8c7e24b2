// The imaging of a whole uneven frame in one persistent launch (FFT form):
// every powfs of the frame -- 32-point sensors and the larger FFT sizes of the
// NGS and tip-tilt sensors -- as one work list of
//
//   WL_N32   a group of 32-point images (one warp each in turn: field, FFT, OTF x uplink x
//            ETF / DTF, inverse, pixels, noise, gradients; ints_n32_kernel's
//            per-warp code),
//   WL_TILE  one tile of one pass of the FFT-pass chain of one large image
//            (gen_pass_kernel's per-tile code),
//   WL_PIX   four large images' pixels, noise and gradients (gen_pixels_item, one
//            warp per image),
//
// taken in list order by resident blocks from a global counter (each block
// fetches its next item while it runs the current one).  The passes of
// one large image depend on one another: each image has a counter of finished
// tiles; a tile of pass p waits (thread 0, bounded) until all tiles of the
// earlier passes are done, and adds one when its own stores are visible.  An
// item waits only on items before it in the list, and those have been handed
// to blocks that run, so the waits end; a wait that exceeds about two seconds
// records SHWFS_ETIMEOUT in the context's error flag and skips the item, and
// every later wait then gives up at once.  The
// list interleaves the passes with slices of the 32-point groups, so the
// large images' chains run beside the 32-point work.  The large images' scratch
// is read from L2 only (L1 is not coherent between the SMs of one launch).
//
// Replaces the per-WFS launch chains of the reference (cuda/sim/wfsgrad.cu:
// 483-745, with per-WFS cuFFT plans, cuda/sim/wfsinit.cu:321-342) by one
// launch for the frame's imaging.
#pragma once
#include "shwfs_gen.cuh"
#include "shwfs_kernels.cuh"

namespace shwfs {

enum WorkType { WL_N32 = 0, WL_TILE = 1, WL_PIX = 2 };
constexpr int WL_THREADS = 128;
constexpr int WL_MAX_SEG = 4;
constexpr long long WL_WAIT_CYCLES = 4000000000LL;  // ~2 s at 1.9 GHz
constexpr int WL_N32_SMEM = 4 * 32 * LD * (int)sizeof(float2);

// One powfs of the frame.
struct WorkSeg {
	PowfsDev P;
	const WfsDev* wfs;
	int nw, nitem;
	int n;         // FFT size: 32, 128 or 256
	int npq;       // pixel slots per lane
	int img0;      // first counter of this powfs's images (large sizes)
	int nt1, ntf;  // tiles of pass 1 and of each later pass
	GenParams G;   // the pass chain of the large sizes
};
struct WorkParams {
	int nseg, nwork;
	WorkSeg seg[WL_MAX_SEG];
	const int4* work;  // (type, segment, first image or item, pass << 16 | tile, or the group's images)
	int* next;         // the dispenser
	int* cnt;          // finished tiles per large image
	int* errflag;
};

__device__ __forceinline__ int wl_ld_acquire(const int* p) {
	int v;
	asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

// Thread 0 waits until *c >= need (bounded); every thread gets the outcome.
__device__ __forceinline__ bool wl_wait(const WorkParams& W, const int* c, int need, int* s_ok) {
	if (threadIdx.x == 0) {
		int ok = 1;
		if (wl_ld_acquire(c) < need) {
			const long long t0 = clock64();
			while (wl_ld_acquire(c) < need) {
				// a wait that expired anywhere ends every later wait at once
				if (clock64() - t0 > WL_WAIT_CYCLES || wl_ld_acquire(W.errflag)) {
					atomicExch(W.errflag, 1);
					ok = 0;
					break;
				}
				__nanosleep(128);
			}
		}
		*s_ok = ok;
	}
	__syncthreads();
	const bool ok = *s_ok != 0;
	// every thread has the outcome before thread 0 may store the next wait's
	// (the pixel items wait on four images in a row)
	__syncthreads();
	return ok;
}

// Tiles of pass p that must be done before it starts (pass 1 none).
__device__ __forceinline__ int wl_need(const WorkSeg& S, int pass) { return pass <= 1 ? 0 : S.nt1 + (pass - 2) * S.ntf; }

// The large images' steps are called out of line, so that their registers do
// not add to the 32-point path's.
template <int N>
__device__ __noinline__ void wl_tile(const WorkSeg& S, int img, int pass, int tile, float2* smem) {
	switch (pass) {
	case GEN_FIELD_COLS: gen_pass_tile<N, GEN_FIELD_COLS, WL_THREADS, true>(S.G, img, tile, smem); break;
	case GEN_PSF_ROWS: gen_pass_tile<N, GEN_PSF_ROWS, WL_THREADS, true>(S.G, img, tile, smem); break;
	case GEN_OTF_COLS: gen_pass_tile<N, GEN_OTF_COLS, WL_THREADS, true>(S.G, img, tile, smem); break;
	default: gen_pass_tile<N, GEN_INV_ROWS, WL_THREADS, true>(S.G, img, tile, smem); break;
	}
}

__device__ __noinline__ void wl_pixels(const WorkSeg& S, int item, int lane) {
	const int n2 = S.n * S.n;
	if (S.npq == 1) gen_pixels_item<1, true>(S.P, S.wfs, S.nw, item, S.G.buf, n2, lane);
	else if (S.npq == 2) gen_pixels_item<2, true>(S.P, S.wfs, S.nw, item, S.G.buf, n2, lane);
	else if (S.npq == 4) gen_pixels_item<4, true>(S.P, S.wfs, S.nw, item, S.G.buf, n2, lane);
	else gen_pixels_item<8, true>(S.P, S.wfs, S.nw, item, S.G.buf, n2, lane);
}

// NPQ: pixel slots per lane of the 32-point items (the largest of the frame's
// 32-point powfs; fewer pixels are handled by the same code).  HALF: the
// 32-point images in the half-spectrum form (the imaging variants 3-5 of
// ints_n32_kernel), else the full-spectrum form, so that the frames equal
// those of the powfs' own launches.
template <int NPQ, bool HALF>
__global__ void __launch_bounds__(WL_THREADS, 4) worklist_kernel(const __grid_constant__ WorkParams W) {
	extern __shared__ float2 wl_s[];
	__shared__ int s_it[2], s_ok;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	if (tid == 0) s_it[0] = atomicAdd(W.next, 1);
	__syncthreads();
	// the next item is fetched while this one runs (a block's reserved item is
	// always later in the list than its current one, so the waits still end)
	for (int par = 0;; par ^= 1) {
		const int it = s_it[par];
		if (it >= W.nwork) break;
		if (tid == 0) s_it[par ^ 1] = atomicAdd(W.next, 1);
		const int4 w = W.work[it];
		const WorkSeg& S = W.seg[w.y];
		if (w.x == WL_N32) {  // w.w images from w.z, one per warp in turn
			const int last = min(S.nitem, w.z + w.w);
			for (int item = w.z + warp; item < last; item += WL_THREADS / 32) {
				const int isa = item / S.nw;
				const WfsDev Wd = S.wfs[item % S.nw];
				float2* tile = wl_s + warp * 32 * LD;
				if (S.P.etfT1) {  // the subaperture's ETF into L2 while the field transforms run
					prefetch_l2(S.P.etfT1 + (size_t)isa * 1024 + 32 * lane);
					prefetch_l2(S.P.etfT1 + (size_t)isa * 1024 + 32 * lane + 16);
				}
				float2 F[32];
				field_fft_n32(Wd.opd + (size_t)isa * 256, Wd.amp + (size_t)isa * 256, S.P.twoinvwvl, tile, lane, F);
				if (HALF) {
					otf_tf_inverse_half_n32(S.P, Wd, isa, lane, tile, F);
					ints_n32_pixels<NPQ>(S.P, Wd, isa, lane, reinterpret_cast<const float*>(tile));
				} else {
					ints_n32_tail<NPQ>(S.P, Wd, isa, lane, tile, F);
				}
			}
		} else if (w.x == WL_TILE) {
			const int pass = w.w >> 16, tile = w.w & 0xffff;
			int* c = W.cnt + S.img0 + w.z;
			if (wl_wait(W, c, wl_need(S, pass), &s_ok)) {
				if (S.n == 128) wl_tile<128>(S, w.z, pass, tile, wl_s);
				else wl_tile<256>(S, w.z, pass, tile, wl_s);
				__threadfence();  // this thread's stores of the tile, before the count
				__syncthreads();
				if (tid == 0) atomicAdd(c, 1);
			}
		} else {  // WL_PIX: four images, each after its whole chain
			const int nimg = min(4, S.nitem - w.z);
			bool ok = true;
			for (int k = 0; k < nimg && ok; k++) ok = wl_wait(W, W.cnt + S.img0 + w.z + k, wl_need(S, GEN_NPASS + 1), &s_ok);
			if (ok && warp < nimg) wl_pixels(S, w.z + warp, lane);
		}
		__syncthreads();  // every thread is done with the shared memory; the next index is in
	}
}

}  // namespace shwfs
