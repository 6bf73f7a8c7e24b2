// C ABI of the B200 Shack-Hartmann frame (declared in include/shwfs_b200.h).
//
// The context owns device copies of the static data that the reference
// uploads in gpu_wfsgrad_init (cuda/sim/wfsinit.cu:159-462), the per-WFS
// frame buffers (cuwfs_t, cuda/sim/wfs.h:72-138) and the FP32 screens
// (gpu_atm2gpu, cuda/sim/atm.cu:106).  Host data arrive in FP64 and MAOS
// layouts; the ETF, DTF nominal and uplink OTF are stored transposed
// (fy fastest) so that the imaging kernel reads them coalesced.
#include <cuda_runtime.h>
#include <emmintrin.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <algorithm>
#include <mutex>
#include <vector>
#include "../../include/shwfs_b200.h"
#include "shwfs_kernels.cuh"
#include "shwfs_tc.cuh"
#include "shwfs_gen.cuh"
#include "shwfs_mtch.cuh"
#include "shwfs_worklist.cuh"

using namespace shwfs;

namespace {

template <typename T>
struct DevBuf {
	T* p = nullptr;
	size_t n = 0;
	void free_() {
		if (p) cudaFree(p);
		p = nullptr;
		n = 0;
	}
};

// geometric sensors: ray trace and gradients of the OPD, no imaging
static inline bool is_geom(int gradtype) { return gradtype == SHWFS_GRAD_ZTILT || gradtype == SHWFS_GRAD_GTILT; }

struct PowfsState {
	shwfs_powfs_desc d;
	DevBuf<double> origx, origy;
	DevBuf<float> amp;  // namp*nsa*nopd^2
	int namp = 0;
	DevBuf<float> saa;
	double saasum = 0;  // sum of saa (sigmatch 2 CoG signal level, powfs.saasum)
	DevBuf<float> nominalT;
	int nnominal = 0;
	DevBuf<int> simap_idx;
	DevBuf<float> simap_wt;
	int nsimap = 0;
	DevBuf<float2> etfT[2];
	int etf_dtrat = 0;  // ETF time interpolation period in frames (0: slot 0 alone)
	int dtrat = 1;      // frames integrated per output frame (powfs.dtrat)
	DevBuf<float> lltamp;
	DevBuf<double> lltorig;  // {llt origx, llt origy}
	// imaging-kernel variant chosen by shwfs_autotune: 0-2 full-spectrum, 3-5
	// half-spectrum 32-point transforms; the half-spectrum form at 5 blocks per
	// SM until the autotuner has run
	int variant = 4;
	std::vector<int> simap_idx_h;     // host copies of the pixel map (TC tables)
	std::vector<double> simap_wt_h;
	DevBuf<uint4> tc_bmat;            // tensor-core B operands (bf16 images)
	DevBuf<float2> gen_buf, gen_lbuf, gen_tw;  // generic-size chain: scratch images (WFS, LLT), twiddles
	DevBuf<float2> lotf_flat;         // uplink OTF of a flat LLT wavefront (matched-filter regeneration)
	DevBuf<float2> seotfT;            // short-exposure OTF per subaperture (matched-filter regeneration), transposed
	DevBuf<float> mtch_img, zero_opd;  // i0/gx/gy scratch; zeros for flat wavefronts
	DevBuf<double> mtch_red;          // i0 sum total, max i0 sum (float bits)
	int tc_ready = 0;
	std::vector<double> origx_h, origy_h;
	std::vector<DevBuf<int>> gs0_ptr, gs0_col;  // G-tilt operators in CSR, one per amplitude
	std::vector<DevBuf<float>> gs0_val;
	// wavelength bands (shwfs_powfs_add_band): a band powfs names its main
	// powfs and weight; the main powfs lists its bands
	int band_of = -1;
	double band_wvlwt = 1;
	std::vector<int> bands;
	std::vector<DevBuf<float2>> band_lotf;  // a band's uplink OTF per WFS (by WFS index)
};

struct WfsState {
	shwfs_wfs_desc d;
	int wfsind = 0;  // index among the WFS of its powfs
	DevBuf<float> mtche, i0sum;
	double i0sumsum = 0;
	DevBuf<float> opd, lltopd, ints, grad;
	DevBuf<float2> lotfT;
	DevBuf<float> neasim;  // geometric gradient noise: Cholesky factor, 3 nsa
	DevBuf<double> i1sum;  // sigmatch 2: total intensity of the frame
	uint64_t seed = 1;
	// closed-loop and static OPD terms (shwfs_wfs_set_opd_terms, shwfs_wfs_set_opdadd)
	DevBuf<float> opdadd;     // NCPA surface on the pupil points, or empty
	int use_dm = 0;           // subtract the mirror grids (shwfs_dm_set) from this WFS's OPD
	int has_poly = 0, has_lltpoly = 0;
	double poly[4] = {0, 0, 0, 0};     // c0 + c1 x + c2 y + c3 (x^2 + y^2) on the pupil points
	double lltpoly[4] = {0, 0, 0, 0};  // the same on the LLT pupil (uplink tip/tilt)
	int garena = -1;          // gradient arena chunk holding grad and grad_h (shwfs_ctx::garena)
	float* grad_h = nullptr;  // pinned staging
	float* ints_h = nullptr;
};

struct LayerState {
	shwfs_layer_desc d;
	DevBuf<float> screen;
};

}  // namespace

struct EvlState;  // science-path evaluation (shwfs_evl_host.cuh)

struct shwfs_ctx {
	int device = 0;
	cudaStream_t stream = nullptr;
	cudaStream_t aux = nullptr;          // LLT/uplink work beside the main ray trace
	cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
	std::string err;
	std::vector<PowfsState> powfs;
	std::vector<WfsState> wfs;
	std::vector<LayerState> atm;
	std::vector<LayerState> dm;          // deformable-mirror grids (shwfs_dm_set), traced after the layers
	float* dm_stage = nullptr;           // pinned FP32 staging of the mirror surfaces
	size_t dm_stage_n = 0;
	cudaEvent_t ev_dm = nullptr;         // the last staging copy has left the host buffer
	double dt = 1.0 / 800;
	int form = SHWFS_FORM_FFT;
	DevBuf<WfsDev> wfsdev;  // staging for per-launch WFS descriptors
	std::vector<WfsDev> wfsdev_h;
	// frame path: descriptors that repeat from frame to frame are uploaded once
	// and served from here (no host-to-device copy, nothing to synchronise)
	struct DescCache {
		std::vector<WfsDev> h;
		DevBuf<WfsDev> d;
	};
	std::vector<DescCache> desc_cache;
	int cache_desc = 0;
	// one stream branch per powfs of a frame, forked from and joined to `stream`
	std::vector<cudaStream_t> pstream;
	std::vector<cudaEvent_t> ev_pfork, ev_pjoin;
	// CUDA graph of a frame (shwfs_frame_graph)
	cudaGraphExec_t gexec = nullptr;
	int g_i0 = -1, g_i1 = -1, g_warm = 0;
	int capturing = 0;
	DevBuf<const float*> llt_in;
	DevBuf<float2*> llt_out;
	DevBuf<int> errflag;                 // bounded device waits record expiry here
	int* errflag_h = nullptr;            // pinned copy read by the frame syncs
	int errflag_armed = 0;               // a kernel that can set errflag ran since the last check
	// gradients of the WFS in consecutive slices of a few chunks (device and
	// pinned host at the same offsets), so that a range of WFS crosses to the
	// host in one copy
	struct GradArena {
		DevBuf<float> d;
		float* h = nullptr;
		size_t cap = 0, used = 0;
	};
	std::vector<GradArena> garena;
	uint64_t h2d_bytes = 0, d2h_bytes = 0;
	// stage timing
	int profiling = 0;
	int trace_order = SHWFS_TRACE_AUTO;  // pupil order of ray-trace launches
	std::vector<cudaEvent_t> ev_pool;
	struct Mark {
		int stage;
		cudaEvent_t a, b;
	};
	std::vector<Mark> marks;
	EvlState* evl = nullptr;
	int sig2_inner = 0;        // launch_ints_sig2 is running the imaging part
	// one persistent imaging launch per frame over a work list (shwfs_set_worklist)
	int worklist = 0;
	int wl_slices = 7;                   // slices of 32-point groups between the passes of the large images
	int wl_group = 4;                    // 32-point images per work item
	int branch_priority = 1;             // the smaller powfs' branches at the greatest stream priority
	int priority = 0;                    // stream priority of the context (shwfs_set_stream_priority)
	struct WorkCache {
		std::vector<int4> h;
		DevBuf<int4> d;
	};
	std::vector<WorkCache> wl_cache;
	DevBuf<int> wl_cnt;                  // dispenser + per-image tile counters
	int dtrat_inner = 0;       // launch_ints_dtrat is running the imaging part
	int band_inner = 0;        // launch_ints_bands is running one band
	int band_accum = 0;        // the band adds to the intensities of the bands before it
};
static void evl_free(shwfs_ctx* ctx);

static cudaEvent_t ev_get(shwfs_ctx* ctx) {
	if (!ctx->ev_pool.empty()) {
		cudaEvent_t e = ctx->ev_pool.back();
		ctx->ev_pool.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}
// Brackets one launch with events when profiling is on.
struct StageMark {
	shwfs_ctx* ctx;
	int stage;
	cudaStream_t st;
	cudaEvent_t a = nullptr;
	StageMark(shwfs_ctx* c, int s, cudaStream_t stream = nullptr) : ctx(c), stage(s), st(stream ? stream : c->stream) {
		if (ctx->profiling) {
			a = ev_get(ctx);
			cudaEventRecord(a, st);
		}
	}
	~StageMark() {
		if (a) {
			cudaEvent_t b = ev_get(ctx);
			cudaEventRecord(b, st);
			ctx->marks.push_back({stage, a, b});
		}
	}
};

static int fail(shwfs_ctx* c, int code, const char* fmt, ...) {
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	if (c) c->err = buf;
	return code;
}
#define CK(call)                                                                                        \
	do {                                                                                                \
		cudaError_t e_ = (call);                                                                        \
		if (e_ != cudaSuccess) return fail(ctx, SHWFS_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
	} while (0)

template <typename T>
static int dev_alloc(shwfs_ctx* ctx, DevBuf<T>& b, size_t n) {
	if (b.n == n && b.p) return 0;
	b.free_();
	if (n == 0) return 0;
	cudaError_t e = cudaMalloc(&b.p, n * sizeof(T));
	if (e != cudaSuccess) {
		b.p = nullptr;
		return fail(ctx, SHWFS_ENOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
	}
	b.n = n;
	return 0;
}
template <typename T>
static int dev_copy(shwfs_ctx* ctx, DevBuf<T>& dst, const DevBuf<T>& src) {
	if (!src.p) {
		dst.free_();
		return 0;
	}
	int r = dev_alloc(ctx, dst, src.n);
	if (r) return r;
	CK(cudaMemcpyAsync(dst.p, src.p, src.n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
	return 0;
}

template <typename T>
static int dev_upload(shwfs_ctx* ctx, DevBuf<T>& b, const T* h, size_t n) {
	int r = dev_alloc(ctx, b, n);
	if (r) return r;
	CK(cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return 0;
}
static int dev_upload_f(shwfs_ctx* ctx, DevBuf<float>& b, const double* h, size_t n) {
	std::vector<float> t(n);
	for (size_t i = 0; i < n; i++) t[i] = (float)h[i];
	return dev_upload(ctx, b, t.data(), n);
}

// FP32 -> FP64 copy of host results (gradients, intensities) with SSE2
// conversions, four values per step.
static void f32_to_f64(const float* __restrict__ src, double* __restrict__ dst, size_t n) {
	size_t k = 0;
	for (; k + 4 <= n; k += 4) {
		const __m128 v = _mm_loadu_ps(src + k);
		_mm_storeu_pd(dst + k, _mm_cvtps_pd(v));
		_mm_storeu_pd(dst + k + 2, _mm_cvtps_pd(_mm_movehl_ps(v, v)));
	}
	for (; k < n; k++) dst[k] = src[k];
}

static int check_errflag(shwfs_ctx* ctx) {
	if (!ctx->errflag.p || !ctx->errflag_armed) return 0;
	ctx->errflag_armed = 0;
	int v = 0;
	CK(cudaMemcpy(&v, ctx->errflag.p, sizeof(int), cudaMemcpyDeviceToHost));
	if (v) {
		CK(cudaMemset(ctx->errflag.p, 0, sizeof(int)));
		return fail(ctx, SHWFS_ETIMEOUT, "a bounded device wait expired in an imaging kernel");
	}
	return 0;
}

static int set_device(shwfs_ctx* ctx) {
	CK(cudaSetDevice(ctx->device));
	return 0;
}

extern "C" {

const char* shwfs_version(void) { return "shwfs_b200 1.0 (sm_100a)"; }

int shwfs_create(shwfs_ctx** pctx, int device) {
	if (!pctx) return SHWFS_EINVAL;
	*pctx = nullptr;
	shwfs_ctx* ctx = new shwfs_ctx();
	ctx->device = device;
	int ndev = 0;
	cudaError_t e = cudaGetDeviceCount(&ndev);
	if (e != cudaSuccess || device < 0 || device >= ndev) {
		delete ctx;
		return SHWFS_ECUDA;
	}
	int prio_lo = 0, prio_hi = 0;
	if (cudaSetDevice(device) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess ||
		cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
		cudaStreamCreateWithPriority(&ctx->aux, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
		cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
		cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess) {
		delete ctx;
		return SHWFS_ECUDA;
	}
	// the log-factorial table of the Poisson sampler, once per device
	{
		static std::mutex mu;
		static bool done[64] = {false};
		std::lock_guard<std::mutex> lock(mu);
		if (device >= 64 || !done[device]) {
			static float t[SHWFS_LOGFACT_N];
			for (int k = 0; k < SHWFS_LOGFACT_N; k++) t[k] = (float)lgamma(k + 1.0);
			if (cudaMemcpyToSymbol(g_logfact, t, sizeof(t)) != cudaSuccess) {
				delete ctx;
				return SHWFS_ECUDA;
			}
			if (device < 64) done[device] = true;
		}
	}
	*pctx = ctx;
	return 0;
}

int shwfs_destroy(shwfs_ctx* ctx) {
	if (!ctx) return SHWFS_EINVAL;
	cudaSetDevice(ctx->device);
	cudaStreamSynchronize(ctx->stream);
	for (auto& p : ctx->powfs) {
		p.origx.free_();
		p.origy.free_();
		p.amp.free_();
		p.saa.free_();
		p.nominalT.free_();
		p.simap_idx.free_();
		p.simap_wt.free_();
		p.etfT[0].free_();
		p.etfT[1].free_();
		p.lltamp.free_();
		p.lltorig.free_();
		p.tc_bmat.free_();
		p.gen_buf.free_();
		p.gen_lbuf.free_();
		p.gen_tw.free_();
		p.lotf_flat.free_();
		p.seotfT.free_();
		p.mtch_img.free_();
		p.zero_opd.free_();
		p.mtch_red.free_();
		for (auto& b : p.gs0_ptr) b.free_();
		for (auto& b : p.gs0_col) b.free_();
		for (auto& b : p.gs0_val) b.free_();
		for (auto& b : p.band_lotf) b.free_();
	}
	evl_free(ctx);
	for (auto& c : ctx->desc_cache) c.d.free_();
	for (auto& c : ctx->wl_cache) c.d.free_();
	ctx->wl_cnt.free_();
	if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
	for (size_t i = 0; i < ctx->pstream.size(); i++) {
		cudaStreamSynchronize(ctx->pstream[i]);
		cudaStreamDestroy(ctx->pstream[i]);
		cudaEventDestroy(ctx->ev_pfork[i]);
		cudaEventDestroy(ctx->ev_pjoin[i]);
	}
	for (auto& w : ctx->wfs) {
		w.mtche.free_();
		w.i0sum.free_();
		w.opd.free_();
		w.lltopd.free_();
		w.ints.free_();
		if (w.garena < 0) {
			w.grad.free_();
			if (w.grad_h) cudaFreeHost(w.grad_h);
		}
		w.lotfT.free_();
		w.neasim.free_();
		w.i1sum.free_();
		if (w.ints_h) cudaFreeHost(w.ints_h);
	}
	for (auto& g : ctx->garena) {
		g.d.free_();
		if (g.h) cudaFreeHost(g.h);
	}
	if (ctx->errflag_h) cudaFreeHost(ctx->errflag_h);
	for (auto& l : ctx->atm) l.screen.free_();
	for (auto& l : ctx->dm) l.screen.free_();
	if (ctx->dm_stage) cudaFreeHost(ctx->dm_stage);
	if (ctx->ev_dm) cudaEventDestroy(ctx->ev_dm);
	for (auto& w : ctx->wfs) w.opdadd.free_();
	for (auto& m : ctx->marks) {
		cudaEventDestroy(m.a);
		cudaEventDestroy(m.b);
	}
	for (auto e : ctx->ev_pool) cudaEventDestroy(e);
	ctx->wfsdev.free_();
	ctx->errflag.free_();
	ctx->llt_in.free_();
	ctx->llt_out.free_();
	cudaStreamSynchronize(ctx->aux);
	cudaEventDestroy(ctx->ev_fork);
	cudaEventDestroy(ctx->ev_join);
	cudaStreamDestroy(ctx->aux);
	cudaStreamDestroy(ctx->stream);
	delete ctx;
	return 0;
}

const char* shwfs_last_error(const shwfs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* shwfs_stream(shwfs_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int shwfs_set_form(shwfs_ctx* ctx, int form) {
	if (!ctx) return SHWFS_EINVAL;
	if (form != SHWFS_FORM_FFT && form != SHWFS_FORM_TC) return fail(ctx, SHWFS_EINVAL, "unknown form %d", form);
	ctx->form = form;
	return 0;
}
int shwfs_set_dt(shwfs_ctx* ctx, double dt) {
	if (!ctx || !(dt > 0)) return SHWFS_EINVAL;
	ctx->dt = dt;
	return 0;
}

int shwfs_powfs_add(shwfs_ctx* ctx, const shwfs_powfs_desc* d, int* ipowfs) {
	if (!ctx || !d || !ipowfs) return SHWFS_EINVAL;
	if (is_geom(d->gradtype)) {
		// geometric sensor: ray trace and z-tilt only, no imaging
		if (d->nsa <= 0 || d->nopd <= 0 || d->nopd > 128)
			return fail(ctx, SHWFS_EINVAL, "powfs: geometric sensor needs nsa > 0 and 0 < nopd <= 128");
		if (d->has_llt) return fail(ctx, SHWFS_EINVAL, "powfs: geometric sensor has no LLT uplink");
		int r = set_device(ctx);
		if (r) return r;
		ctx->powfs.emplace_back();
		shwfs_powfs_desc& g = ctx->powfs.back().d;
		g = *d;
		g.pixpsax = g.pixpsay = 0;  // no detector
		g.has_etf = 0;
		*ipowfs = (int)ctx->powfs.size() - 1;
		return 0;
	}
	if (d->nsa <= 0 || d->nopd <= 0 || d->embfac <= 0 || d->notf <= 0 || d->pixpsax <= 0 || d->pixpsay <= 0)
		return fail(ctx, SHWFS_EINVAL, "powfs: sizes must be positive");
	const int nw = d->nopd * d->embfac;
	const bool n32 = d->nopd == 16 && nw == 32 && d->notf == 32;
	const bool gen = nw == d->notf && (d->notf == 64 || d->notf == 128 || d->notf == 256);
	if (!n32 && !gen)
		return fail(ctx, SHWFS_EINVAL,
			"powfs: n_opd=%d n_w=%d n_f=%d not supported by this build (16/32/32, or n_w = n_f in {64, 128, 256})",
			d->nopd, nw, d->notf);
	if (d->pixpsax * d->pixpsay > (n32 ? 128 : 256))
		return fail(ctx, SHWFS_EINVAL, "powfs: at most %d pixels per subaperture", n32 ? 128 : 256);
	if (d->gradtype != SHWFS_GRAD_MF && d->gradtype != SHWFS_GRAD_COG)
		return fail(ctx, SHWFS_EINVAL, "powfs: gradtype must be SHWFS_GRAD_MF, SHWFS_GRAD_COG, SHWFS_GRAD_ZTILT or SHWFS_GRAD_GTILT");
	if (d->sigmatch < 0 || d->sigmatch > 2) return fail(ctx, SHWFS_EINVAL, "powfs: sigmatch must be 0, 1 or 2");
	if (d->has_llt && d->llt_nx != d->nopd)
		return fail(ctx, SHWFS_EINVAL, "powfs: LLT pupil sampling (%d) must equal the subaperture's (%d)", d->llt_nx, d->nopd);
	if (d->has_llt && d->llt_nx * d->embfac != d->notf)
		return fail(ctx, SHWFS_EINVAL, "powfs: LLT pupil of %d points is not supported (needs %d)", d->llt_nx,
			d->notf / d->embfac);
	int r = set_device(ctx);
	if (r) return r;
	ctx->powfs.emplace_back();
	ctx->powfs.back().d = *d;
	*ipowfs = (int)ctx->powfs.size() - 1;
	return 0;
}

static PowfsState* get_powfs(shwfs_ctx* ctx, int ipowfs) {
	if (!ctx || ipowfs < 0 || ipowfs >= (int)ctx->powfs.size()) return nullptr;
	return &ctx->powfs[ipowfs];
}
static WfsState* get_wfs(shwfs_ctx* ctx, int iwfs) {
	if (!ctx || iwfs < 0 || iwfs >= (int)ctx->wfs.size()) return nullptr;
	return &ctx->wfs[iwfs];
}

int shwfs_powfs_set_geom(shwfs_ctx* ctx, int ipowfs, const double* origx, const double* origy, const double* amp,
	int namp, const double* saa) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || !origx || !origy || !amp || namp <= 0) return ctx ? fail(ctx, SHWFS_EINVAL, "set_geom: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const int nsa = p->d.nsa, n2 = p->d.nopd * p->d.nopd;
	p->origx_h.assign(origx, origx + nsa);
	p->origy_h.assign(origy, origy + nsa);
	if ((r = dev_upload(ctx, p->origx, origx, nsa))) return r;
	if ((r = dev_upload(ctx, p->origy, origy, nsa))) return r;
	if ((r = dev_upload_f(ctx, p->amp, amp, (size_t)namp * nsa * n2))) return r;
	p->namp = namp;
	p->saasum = nsa;
	if (saa) {
		if ((r = dev_upload_f(ctx, p->saa, saa, nsa))) return r;
		p->saasum = 0;
		for (int i = 0; i < nsa; i++) p->saasum += saa[i];
	}
	return 0;
}

// transpose each notf x notf block: out[fy + n*fx] = in[fx + n*fy]
static void transpose_blocks_real(const double* in, float* out, int nblk, int n) {
	for (int b = 0; b < nblk; b++)
		for (int fy = 0; fy < n; fy++)
			for (int fx = 0; fx < n; fx++) out[(size_t)b * n * n + fy + n * fx] = (float)in[(size_t)b * n * n + fx + n * fy];
}
static void transpose_blocks_cplx(const double* in, float2* out, int nblk, int n) {
	for (int b = 0; b < nblk; b++)
		for (int fy = 0; fy < n; fy++)
			for (int fx = 0; fx < n; fx++) {
				const size_t i = (size_t)b * n * n + fx + n * fy;
				out[(size_t)b * n * n + fy + n * fx] = make_float2((float)in[2 * i], (float)in[2 * i + 1]);
			}
}

int shwfs_powfs_set_nominal(shwfs_ctx* ctx, int ipowfs, const double* nominal, int nnominal) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || !nominal || (nnominal != 1 && nnominal != p->d.nsa))
		return ctx ? fail(ctx, SHWFS_EINVAL, "set_nominal: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const int n = p->d.notf;
	std::vector<float> t((size_t)nnominal * n * n);
	transpose_blocks_real(nominal, t.data(), nnominal, n);
	if ((r = dev_upload(ctx, p->nominalT, t.data(), t.size()))) return r;
	p->nnominal = nnominal;
	return 0;
}

int shwfs_powfs_set_simap(shwfs_ctx* ctx, int ipowfs, const int* idx, const double* wt, int nmap) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || !idx || !wt || (nmap != 1 && nmap != p->d.nsa)) return ctx ? fail(ctx, SHWFS_EINVAL, "set_simap: bad arguments") : SHWFS_EINVAL;
	const int npix = p->d.pixpsax * p->d.pixpsay, n2 = p->d.notf * p->d.notf;
	const size_t m = (size_t)nmap * npix * 4;
	for (size_t i = 0; i < m; i++) {
		if (idx[i] < -1 || idx[i] >= n2) return fail(ctx, SHWFS_EINVAL, "set_simap: index %d out of [-1,%d)", idx[i], n2);
	}
	int r = set_device(ctx);
	if (r) return r;
	// a missing tap (index -1) carries weight 0, whatever the caller left there:
	// the sampling kernels multiply it by 0 instead of branching around it
	std::vector<float> w(m);
	for (size_t i = 0; i < m; i++) w[i] = idx[i] < 0 ? 0.f : (float)wt[i];
	if ((r = dev_upload(ctx, p->simap_idx, idx, m))) return r;
	if ((r = dev_upload(ctx, p->simap_wt, w.data(), m))) return r;
	p->nsimap = nmap;
	p->simap_idx_h.assign(idx, idx + m);
	p->simap_wt_h.assign(wt, wt + m);
	p->tc_ready = 0;
	return 0;
}

int shwfs_powfs_set_etf(shwfs_ctx* ctx, int ipowfs, const double* etf, int slot) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || !etf || slot < 0 || slot > 1) return ctx ? fail(ctx, SHWFS_EINVAL, "set_etf: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const int n = p->d.notf;
	std::vector<float2> t((size_t)p->d.nsa * n * n);
	transpose_blocks_cplx(etf, t.data(), p->d.nsa, n);
	if ((r = dev_upload(ctx, p->etfT[slot], t.data(), t.size()))) return r;
	return 0;
}

int shwfs_powfs_set_seotf(shwfs_ctx* ctx, int ipowfs, const double* seotf) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || is_geom(p->d.gradtype)) return ctx ? fail(ctx, SHWFS_EINVAL, "set_seotf: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (!seotf) {
		CK(cudaStreamSynchronize(ctx->stream));
		p->seotfT.free_();
		return 0;
	}
	const int n = p->d.notf;
	std::vector<float2> t((size_t)p->d.nsa * n * n);
	transpose_blocks_cplx(seotf, t.data(), p->d.nsa, n);
	return dev_upload(ctx, p->seotfT, t.data(), t.size());
}

int shwfs_powfs_set_lltamp(shwfs_ctx* ctx, int ipowfs, const double* lltamp) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || !lltamp || !p->d.has_llt) return ctx ? fail(ctx, SHWFS_EINVAL, "set_lltamp: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const double orig[2] = {p->d.llt_origx, p->d.llt_origy};
	if ((r = dev_upload(ctx, p->lltorig, orig, 2))) return r;
	return dev_upload_f(ctx, p->lltamp, lltamp, (size_t)p->d.llt_nx * p->d.llt_nx);
}

int shwfs_powfs_add_band(shwfs_ctx* ctx, int ipowfs, const shwfs_powfs_desc* d, double wvlwt, int* iband) {
	PowfsState* m = get_powfs(ctx, ipowfs);
	if (!m || !d || !iband || !(wvlwt >= 0)) return ctx ? fail(ctx, SHWFS_EINVAL, "add_band: bad arguments") : SHWFS_EINVAL;
	if (m->band_of >= 0) return fail(ctx, SHWFS_EINVAL, "add_band: powfs %d is itself a band", ipowfs);
	if (is_geom(m->d.gradtype)) return fail(ctx, SHWFS_EINVAL, "add_band: a geometric sensor forms no images");
	if (m->bands.size() >= SHWFS_MAX_BANDS) return fail(ctx, SHWFS_EINVAL, "add_band: at most %d bands", SHWFS_MAX_BANDS);
	if (!m->amp.p || !m->origx.p) return fail(ctx, SHWFS_ESTATE, "add_band: set the geometry of powfs %d first", ipowfs);
	const shwfs_powfs_desc& a = m->d;
	if (d->nsa != a.nsa || d->nopd != a.nopd || d->embfac != a.embfac || d->notf != a.notf || d->pixpsax != a.pixpsax ||
		d->pixpsay != a.pixpsay || d->has_etf != a.has_etf || d->has_llt != a.has_llt || d->llt_nx != a.llt_nx ||
		d->gradtype != a.gradtype || d->sigmatch != a.sigmatch || d->dsa != a.dsa || d->dx != a.dx || !(d->wvl > 0))
		return fail(ctx, SHWFS_EINVAL,
			"add_band: a band keeps its powfs' subapertures, sampling, sizes, pixels, LLT and gradient options; only the "
			"wavelength and the transfer functions differ");
	int ib = -1, r = shwfs_powfs_add(ctx, d, &ib);
	if (r) return r;
	PowfsState& M = ctx->powfs[ipowfs];  // the powfs vector may have grown
	PowfsState& B = ctx->powfs[ib];
	B.band_of = ipowfs;
	B.band_wvlwt = wvlwt;
	// the band images the main powfs' subapertures: its geometry, as set now
	if ((r = dev_copy(ctx, B.origx, M.origx)) || (r = dev_copy(ctx, B.origy, M.origy)) ||
		(r = dev_copy(ctx, B.amp, M.amp)) || (r = dev_copy(ctx, B.saa, M.saa)) ||
		(r = dev_copy(ctx, B.lltamp, M.lltamp)) || (r = dev_copy(ctx, B.lltorig, M.lltorig)))
		return r;
	CK(cudaStreamSynchronize(ctx->stream));
	B.namp = M.namp;
	B.saasum = M.saasum;
	B.origx_h = M.origx_h;
	B.origy_h = M.origy_h;
	B.dtrat = 1;
	M.bands.push_back(ib);
	*iband = ib;
	return 0;
}

int shwfs_wfs_add(shwfs_ctx* ctx, const shwfs_wfs_desc* d, int* iwfs) {
	if (!ctx || !d || !iwfs) return SHWFS_EINVAL;
	PowfsState* p = get_powfs(ctx, d->ipowfs);
	if (!p) return fail(ctx, SHWFS_EINVAL, "wfs_add: unknown powfs %d", d->ipowfs);
	if (p->band_of >= 0)
		return fail(ctx, SHWFS_EINVAL, "wfs_add: powfs %d is a wavelength band of powfs %d; add the WFS there", d->ipowfs,
			p->band_of);
	int r = set_device(ctx);
	if (r) return r;
	ctx->wfs.emplace_back();
	WfsState& w = ctx->wfs.back();
	w.d = *d;
	int count = 0;
	for (size_t i = 0; i + 1 < ctx->wfs.size(); i++)
		if (ctx->wfs[i].d.ipowfs == d->ipowfs) count++;
	w.wfsind = count;
	const int nsa = p->d.nsa, npix = p->d.pixpsax * p->d.pixpsay;
	if ((r = dev_alloc(ctx, w.opd, (size_t)nsa * p->d.nopd * p->d.nopd))) return r;
	if ((r = dev_alloc(ctx, w.ints, (size_t)nsa * npix))) return r;
	{
		const size_t need = (size_t)2 * nsa;
		if (ctx->garena.empty() || ctx->garena.back().used + need > ctx->garena.back().cap) {
			ctx->garena.emplace_back();
			auto& g = ctx->garena.back();
			g.cap = std::max((size_t)1 << 18, need);
			if ((r = dev_alloc(ctx, g.d, g.cap))) return r;
			CK(cudaMallocHost(&g.h, sizeof(float) * g.cap));
		}
		auto& g = ctx->garena.back();
		w.garena = (int)ctx->garena.size() - 1;
		w.grad.p = g.d.p + g.used;
		w.grad.n = need;
		w.grad_h = g.h + g.used;
		g.used += need;
	}
	CK(cudaMemsetAsync(w.grad.p, 0, sizeof(float) * 2 * nsa, ctx->stream));
	if (p->d.has_llt) {
		if ((r = dev_alloc(ctx, w.lltopd, (size_t)p->d.llt_nx * p->d.llt_nx))) return r;
		if ((r = dev_alloc(ctx, w.lotfT, (size_t)p->d.notf * p->d.notf))) return r;
	}
	if (npix > 0) CK(cudaMallocHost(&w.ints_h, sizeof(float) * nsa * npix));
	CK(cudaStreamSynchronize(ctx->stream));
	*iwfs = (int)ctx->wfs.size() - 1;
	return 0;
}

int shwfs_wfs_set_mtche(shwfs_ctx* ctx, int iwfs, const double* mtche, const double* i0sum, double i0sumsum) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "set_mtche: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	const int nsa = p.d.nsa, npix = p.d.pixpsax * p.d.pixpsay;
	int r = set_device(ctx);
	if (r) return r;
	if (mtche && (r = dev_upload_f(ctx, w->mtche, mtche, (size_t)nsa * 2 * npix))) return r;
	if (i0sum && (r = dev_upload_f(ctx, w->i0sum, i0sum, nsa))) return r;
	w->i0sumsum = i0sumsum;
	return 0;
}

int shwfs_wfs_get_mtche(shwfs_ctx* ctx, int iwfs, double* mtche, double* i0sum, double* i0sumsum) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "get_mtche: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	const size_t nsa = p.d.nsa, n = nsa * 2 * p.d.pixpsax * p.d.pixpsay;
	if ((mtche && !w->mtche.p) || (i0sum && !w->i0sum.p))
		return fail(ctx, SHWFS_ESTATE, "get_mtche: WFS %d has no matched filter", iwfs);
	int r = set_device(ctx);
	if (r) return r;
	std::vector<float> t(std::max(n, nsa));
	if (mtche) {
		CK(cudaMemcpyAsync(t.data(), w->mtche.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
		for (size_t k = 0; k < n; k++) mtche[k] = t[k];
	}
	if (i0sum) {
		CK(cudaMemcpyAsync(t.data(), w->i0sum.p, nsa * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
		for (size_t k = 0; k < nsa; k++) i0sum[k] = t[k];
	}
	if (i0sumsum) *i0sumsum = w->i0sumsum;
	return 0;
}

int shwfs_wfs_seed(shwfs_ctx* ctx, int iwfs, uint64_t seed) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "wfs_seed: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	w->seed = seed;
	return 0;
}

int shwfs_atm_set(shwfs_ctx* ctx, int nlayer, const shwfs_layer_desc* layers, const double* const* screens) {
	if (!ctx || nlayer < 0 || nlayer > SHWFS_MAX_LAYERS || (nlayer && (!layers || !screens)))
		return ctx ? fail(ctx, SHWFS_EINVAL, "atm_set: 0..%d layers", SHWFS_MAX_LAYERS) : SHWFS_EINVAL;
	if (nlayer + (int)ctx->dm.size() > SHWFS_MAX_LAYERS)
		return fail(ctx, SHWFS_EINVAL, "atm_set: %d layers and %d mirror grids exceed %d", nlayer, (int)ctx->dm.size(),
			SHWFS_MAX_LAYERS);
	int r = set_device(ctx);
	if (r) return r;
	for (auto& l : ctx->atm) l.screen.free_();
	ctx->atm.clear();
	ctx->atm.resize(nlayer);
	for (int i = 0; i < nlayer; i++) {
		if (layers[i].nx < 2 || layers[i].ny < 2 || !(layers[i].dx > 0) || !screens[i])
			return fail(ctx, SHWFS_EINVAL, "atm_set: layer %d is invalid", i);
		ctx->atm[i].d = layers[i];
		if ((r = dev_upload_f(ctx, ctx->atm[i].screen, screens[i], (size_t)layers[i].nx * layers[i].ny))) return r;
	}
	return 0;
}

int shwfs_dm_set(shwfs_ctx* ctx, int ndm, const shwfs_layer_desc* dms, const double* const* surfaces) {
	if (!ctx || ndm < 0 || (ndm && (!dms || !surfaces))) return ctx ? fail(ctx, SHWFS_EINVAL, "dm_set: bad arguments") : SHWFS_EINVAL;
	if ((int)ctx->atm.size() + ndm > SHWFS_MAX_LAYERS)
		return fail(ctx, SHWFS_EINVAL, "dm_set: %d layers and %d mirror grids exceed %d", (int)ctx->atm.size(), ndm,
			SHWFS_MAX_LAYERS);
	size_t total = 0;
	for (int i = 0; i < ndm; i++) {
		const shwfs_layer_desc& d = dms[i];
		if (d.nx < 2 || d.ny < 2 || !(d.dx > 0) || !surfaces[i] || !isfinite(d.ht) || !isfinite(d.alpha))
			return fail(ctx, SHWFS_EINVAL, "dm_set: mirror %d is invalid", i);
		total += (size_t)d.nx * d.ny;
	}
	int r = set_device(ctx);
	if (r) return r;
	if (!ctx->ev_dm) CK(cudaEventCreateWithFlags(&ctx->ev_dm, cudaEventDisableTiming));
	// the previous frame's surfaces may still be on their way out of the staging buffer
	CK(cudaEventSynchronize(ctx->ev_dm));
	if (ndm == 0) {
		for (auto& m : ctx->dm) m.screen.free_();
		ctx->dm.clear();
		return 0;
	}
	if ((int)ctx->dm.size() != ndm) {
		for (auto& m : ctx->dm) m.screen.free_();
		ctx->dm.clear();
		ctx->dm.resize(ndm);
	}
	if (ctx->dm_stage_n < total) {
		if (ctx->dm_stage) cudaFreeHost(ctx->dm_stage);
		ctx->dm_stage = nullptr;
		ctx->dm_stage_n = 0;
		CK(cudaMallocHost(&ctx->dm_stage, total * sizeof(float)));
		ctx->dm_stage_n = total;
	}
	size_t off = 0;
	for (int i = 0; i < ndm; i++) {
		const size_t n = (size_t)dms[i].nx * dms[i].ny;
		if ((r = dev_alloc(ctx, ctx->dm[i].screen, n))) return r;
		ctx->dm[i].d = dms[i];
		float* st = ctx->dm_stage + off;
		for (size_t k = 0; k < n; k++) st[k] = (float)surfaces[i][k];
		CK(cudaMemcpyAsync(ctx->dm[i].screen.p, st, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
		ctx->h2d_bytes += n * sizeof(float);
		off += n;
	}
	CK(cudaEventRecord(ctx->ev_dm, ctx->stream));
	return 0;
}

int shwfs_wfs_set_opd_terms(shwfs_ctx* ctx, int iwfs, int use_dm, const double* ptt, double focus_tel,
	double focus_llt, const double* lltptt) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "set_opd_terms: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	const PowfsState& p = ctx->powfs[w->d.ipowfs];
	if (lltptt && (lltptt[0] != 0 || lltptt[1] != 0) && !p.d.has_llt)
		return fail(ctx, SHWFS_EINVAL, "set_opd_terms: LLT tip/tilt for WFS %d, whose powfs has no LLT", iwfs);
	const double t0 = ptt ? ptt[0] : 0, t1 = ptt ? ptt[1] : 0, t2 = ptt ? ptt[2] : 0;
	if (!isfinite(t0) || !isfinite(t1) || !isfinite(t2) || !isfinite(focus_tel) || !isfinite(focus_llt))
		return fail(ctx, SHWFS_EINVAL, "set_opd_terms: terms must be finite");
	if ((focus_tel != 0 || focus_llt != 0) && p.origx_h.empty())
		return fail(ctx, SHWFS_ESTATE, "set_opd_terms: powfs geometry not set");
	w->use_dm = use_dm ? 1 : 0;
	// loc_add_ptt (math/loc.c:762-789): ptt[0] + ptt[1] x + ptt[2] y.
	// loc_add_focus_offset (math/loc.c:1226-1246): f ((x-a)^2 + (y-b)^2) less its
	// mean over the pupil points, for the telescope focus (a = b = 0) and the LLT
	// zoom focus (a, b = the LLT position); expanded about the origin in FP64.
	double c[4] = {t0, t1, t2, focus_tel + focus_llt};
	if (focus_tel != 0 || focus_llt != 0) {
		const int nopd = p.d.nopd;
		const double n = (double)p.d.nsa * nopd * nopd;
		double sx = 0, sy = 0, sr = 0;
		for (int isa = 0; isa < p.d.nsa; isa++)
			for (int iy = 0; iy < nopd; iy++)
				for (int ix = 0; ix < nopd; ix++) {
					const double x = p.origx_h[isa] + ix * p.d.dx, y = p.origy_h[isa] + iy * p.d.dx;
					sx += x;
					sy += y;
					sr += x * x + y * y;
				}
		const double a = p.d.llt_ox, b = p.d.llt_oy;
		c[0] -= focus_tel * sr / n;
		c[0] += focus_llt * (a * a + b * b) - focus_llt * (sr - 2 * a * sx - 2 * b * sy + n * (a * a + b * b)) / n;
		c[1] -= 2 * focus_llt * a;
		c[2] -= 2 * focus_llt * b;
	}
	w->has_poly = c[0] != 0 || c[1] != 0 || c[2] != 0 || c[3] != 0;
	memcpy(w->poly, c, sizeof(c));
	w->lltpoly[0] = 0;
	w->lltpoly[1] = lltptt ? lltptt[0] : 0;
	w->lltpoly[2] = lltptt ? lltptt[1] : 0;
	w->lltpoly[3] = 0;
	w->has_lltpoly = w->lltpoly[1] != 0 || w->lltpoly[2] != 0;
	return 0;
}

int shwfs_wfs_set_opdadd(shwfs_ctx* ctx, int iwfs, const double* opd) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "set_opdadd: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (!opd) {
		CK(cudaStreamSynchronize(ctx->stream));
		w->opdadd.free_();
		return 0;
	}
	const PowfsState& p = ctx->powfs[w->d.ipowfs];
	return dev_upload_f(ctx, w->opdadd, opd, (size_t)p.d.nsa * p.d.nopd * p.d.nopd);
}

}  // extern "C"

// ---- frame machinery ----

static int launch_geom_wfs(shwfs_ctx* ctx, GeomParams& gp, bool split = true);
static int sm_count(shwfs_ctx* ctx);

// Appends one pupil to a batched ray-trace launch: per-layer geometry of
// prop_range (lib/accphi.c:223-244) and prop_grid_pts
// (lib/accphi_grid_do.c:408-434), FP64 on the host.
static int add_geom_entry(shwfs_ctx* ctx, GeomParams& gp, double thetax, double thetay, double hs, double hc,
	double misregx, double misregy, double extra_shiftx, double extra_shifty, int isim, const double* origx,
	const double* origy, int nsa, int nopd, double dx, float* out, bool mirrors = false) {
	if (gp.nentry >= SHWFS_MAX_ENTRIES) return fail(ctx, SHWFS_EINVAL, "too many pupils in one ray-trace launch");
	GeomEntry& e = gp.e[gp.nentry++];
	memset(&e, 0, sizeof(e));
	e.origx = origx;
	e.origy = origy;
	e.opd = out;
	e.nsa = nsa;
	e.nopd = nopd;
	e.dx = dx;
	e.use = 0;
	for (int l = 0; l < (int)ctx->atm.size(); l++) {
		const shwfs_layer_desc& a = ctx->atm[l].d;
		const double ht = a.ht;
		const bool finite_hs = isfinite(hs) && hs != 0;
		if (finite_hs && (hc > hs || ht > hs)) continue;
		const double scale = finite_hs ? 1. - (ht - hc) / (hs - hc) : 1.;
		if (scale < 0) continue;
		const double shiftx = -a.vx * ctx->dt * isim + extra_shiftx;
		const double shifty = -a.vy * ctx->dt * isim + extra_shifty;
		const double displacex = ht * thetax + scale * misregx + shiftx;
		const double displacey = ht * thetay + scale * misregy + shifty;
		const double dx_in1 = 1. / a.dx;
		e.sx[l] = scale * dx_in1;
		e.dispx[l] = (displacex - a.ox) * dx_in1;
		e.dispy[l] = (displacey - a.oy) * dx_in1;
		e.use |= 1u << l;
	}
	// mirror grids after the layers: the WFS's cone, misregistration, no wind
	// (mapcell2loc, cuda/sim/accphi.cu:238-249; maos/sim_utils.c:1034-1052)
	const int na = (int)ctx->atm.size();
	for (int k = 0; mirrors && k < (int)ctx->dm.size(); k++) {
		const shwfs_layer_desc& a = ctx->dm[k].d;
		const int l = na + k;
		const double ht = a.ht;
		const bool finite_hs = isfinite(hs) && hs != 0;
		const double scale = finite_hs ? 1. - (ht - hc) / (hs - hc) : 1.;
		if (scale < 0) continue;
		const double dx_in1 = 1. / a.dx;
		e.sx[l] = scale * dx_in1;
		e.dispx[l] = (ht * thetax + scale * misregx - a.ox) * dx_in1;
		e.dispy[l] = (ht * thetay + scale * misregy - a.oy) * dx_in1;
		e.use |= 1u << l;
	}
	return 0;
}

static void geom_init(shwfs_ctx* ctx, GeomParams& gp) {
	memset(&gp, 0, sizeof(gp));
	gp.nlayer = (int)ctx->atm.size();
	for (int l = 0; l < gp.nlayer; l++) {
		gp.screen[l] = ctx->atm[l].screen.p;
		gp.nx[l] = (int)ctx->atm[l].d.nx;
		gp.ny[l] = (int)ctx->atm[l].d.ny;
		gp.alpha[l] = (float)ctx->atm[l].d.alpha;
	}
	for (const LayerState& m : ctx->dm) {  // mirror grids last (shwfs_dm_set)
		const int l = gp.nlayer++;
		gp.screen[l] = m.screen.p;
		gp.nx[l] = (int)m.d.nx;
		gp.ny[l] = (int)m.d.ny;
		gp.alpha[l] = (float)m.d.alpha;
		gp.nmirror++;
	}
}

// LLT pupils go to llt_uplink_kernel on the aux stream (forked from and
// joined back into the main stream); subaperture pupils to geom_kernel.
static int launch_geom(shwfs_ctx* ctx, GeomParams& all) {
	GeomParams gp, lp;
	memcpy(&gp, &all, sizeof(GeomParams));
	memcpy(&lp, &all, sizeof(GeomParams));
	gp.nentry = lp.nentry = 0;
	for (int i = 0; i < all.nentry; i++) {
		if (all.e[i].lltamp) lp.e[lp.nentry++] = all.e[i];
		else gp.e[gp.nentry++] = all.e[i];
	}
	// the subaperture trace (the frame's critical path) is launched first; the
	// uplink follows on the aux stream, whose greater priority lets its few
	// blocks start as the trace's first blocks retire
	if (lp.nentry) CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
	int r = launch_geom_wfs(ctx, gp);
	if (lp.nentry) {
		CK(cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0));
		{
			StageMark m(ctx, SHWFS_STAGE_UPLINK, ctx->aux);
			llt_uplink_kernel<<<lp.nentry, 256, 0, ctx->aux>>>(lp);
		}
		CK(cudaGetLastError());
		CK(cudaEventRecord(ctx->ev_join, ctx->aux));
		CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
	}
	return r;
}


static int l2_bytes(shwfs_ctx* ctx) {
	static int l2[64] = {0};
	if (ctx->device < 64 && l2[ctx->device]) return l2[ctx->device];
	int v = 0;
	cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, ctx->device);
	if (v <= 0) v = 126 << 20;
	if (ctx->device < 64) l2[ctx->device] = v;
	return v;
}

// The open-loop trace kernel for 16x16 or 32x32 pupils and 1-8 layers (their
// tables stay below the 48 KB default of dynamic shared memory).
using GeomKernel = void (*)(const GeomParams, int, int, int);
template <int NOPD>
static GeomKernel geom_pick_n(int nl) {
	switch (nl) {
	case 1: return geom_kernel<false, NOPD, 1>;
	case 2: return geom_kernel<false, NOPD, 2>;
	case 3: return geom_kernel<false, NOPD, 3>;
	case 4: return geom_kernel<false, NOPD, 4>;
	case 5: return geom_kernel<false, NOPD, 5>;
	case 6: return geom_kernel<false, NOPD, 6>;
	case 7: return geom_kernel<false, NOPD, 7>;
	case 8: return geom_kernel<false, NOPD, 8>;
	default: return geom_kernel<false, NOPD, 0>;
	}
}
static GeomKernel geom_pick(int nopd, int nl) { return nopd == 16 ? geom_pick_n<16>(nl) : geom_pick_n<32>(nl); }

// split: when the launch's screens exceed L2, the pupils of the largest size
// are traced interleaved (each screen row their footprints share is fetched
// from DRAM once while in L2) and any other pupils in a second launch.  With
// the screens in L2, the order as listed keeps each block's neighbours on the
// same footprint, which measured faster.
static int launch_geom_wfs(shwfs_ctx* ctx, GeomParams& gp, bool split) {
	if (ctx->trace_order == SHWFS_TRACE_LISTED) gp.interleave = 0;
	if (split && !gp.interleave && gp.nentry >= 2 && ctx->trace_order != SHWFS_TRACE_LISTED) {
		double screen = 0;
		for (int l = 0; l < gp.nlayer; l++) screen += 4.0 * gp.nx[l] * gp.ny[l];
		int nmax = 0, nbig = 0;
		for (int i = 0; i < gp.nentry; i++) nmax = std::max(nmax, gp.e[i].nsa);
		for (int i = 0; i < gp.nentry; i++) nbig += gp.e[i].nsa == nmax;
		const bool want = ctx->trace_order == SHWFS_TRACE_INTERLEAVED || screen > l2_bytes(ctx);
		if (want && nbig >= 2) {
			if (nbig == gp.nentry) {
				gp.interleave = 1;
			} else {
				GeomParams big, rest;
				memcpy(&big, &gp, sizeof(GeomParams));
				memcpy(&rest, &gp, sizeof(GeomParams));
				big.nentry = rest.nentry = 0;
				for (int i = 0; i < gp.nentry; i++) {
					if (gp.e[i].nsa == nmax) big.e[big.nentry++] = gp.e[i];
					else rest.e[rest.nentry++] = gp.e[i];
				}
				big.interleave = 1;
				int r = launch_geom_wfs(ctx, big, false);
				return r ? r : launch_geom_wfs(ctx, rest, false);
			}
		}
	}
	int nitem = 0;
	const int nopd = gp.nentry ? gp.e[0].nopd : 0;
	for (int i = 0; i < gp.nentry; i++) {
		if (gp.e[i].nopd != nopd) return fail(ctx, SHWFS_EINVAL, "ray trace: pupils of one launch need the same sampling");
		if (gp.interleave && gp.e[i].nsa != gp.e[0].nsa)
			return fail(ctx, SHWFS_EINVAL, "ray trace: interleaved pupils need the same number of subapertures");
		gp.e[i].item0 = nitem;
		nitem += gp.e[i].nsa;
	}
	if (nitem == 0) return 0;
	const int nblk = nitem;
	if (gp.nlayer == 0) {  // no turbulence: zero OPD and a flat-wavefront uplink
		for (int i = 0; i < gp.nentry; i++)
			if (gp.e[i].opd)
				CK(cudaMemsetAsync(gp.e[i].opd, 0, sizeof(float) * gp.e[i].nsa * gp.e[i].nopd * gp.e[i].nopd, ctx->stream));
	}
	{
		StageMark m(ctx, SHWFS_STAGE_RAYTRACE);
		const size_t smem = (size_t)gp.nlayer * nopd * 2 * sizeof(int4);
		if (smem > 160 * 1024) return fail(ctx, SHWFS_EINVAL, "ray trace: %d layers x %d points too large", gp.nlayer, nopd);
		bool extra = gp.nmirror > 0;
		for (int i = 0; i < gp.nentry; i++) extra = extra || gp.e[i].opdadd || gp.e[i].has_poly;
		if (smem > 48 * 1024) {
			CK(cudaFuncSetAttribute(geom_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
			CK(cudaFuncSetAttribute(geom_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		}
		// GEOM_PTS points per thread with no idle slot where the pupil allows it:
		// 16x16 pupils 64 threads, 32x32 256, larger ones split over blocks of 256
		const int np = nopd * nopd;
		const int bd = std::min(256, std::max(32, ((np + GEOM_PTS - 1) / GEOM_PTS + 31) / 32 * 32));
		int bps = (np + GEOM_PTS * bd - 1) / (GEOM_PTS * bd);  // blocks per subaperture
		const bool fixed = !extra && (nopd == 16 || nopd == 32) && gp.nlayer <= 8;
		gp.ppt = GEOM_PTS;
		if (!fixed && (long)nblk * bps < sm_count(ctx)) {  // a few pupils: a point per thread, more blocks
			gp.ppt = 1;
			bps = (np + bd - 1) / bd;
		}
		if (extra) geom_kernel<true><<<(unsigned)nblk * bps, bd, smem, ctx->stream>>>(gp, nopd, nitem, bps);
		else if (fixed)  // pupil side and layer count fixed at compile time
			geom_pick(nopd, gp.nlayer)<<<(unsigned)nblk * bps, bd, smem, ctx->stream>>>(gp, nopd, nitem, bps);
		else geom_kernel<false><<<(unsigned)nblk * bps, bd, smem, ctx->stream>>>(gp, nopd, nitem, bps);
	}
	CK(cudaGetLastError());
	return 0;
}

// The ray-trace entry of one WFS.
static int add_wfs_entry(shwfs_ctx* ctx, GeomParams& gp, WfsState& w, int isim, float* opd) {
	PowfsState& p = ctx->powfs[w.d.ipowfs];
	int r = add_geom_entry(ctx, gp, w.d.thetax, w.d.thetay, w.d.hs, w.d.hc, w.d.misregx, w.d.misregy, 0, 0, isim,
		p.origx.p, p.origy.p, p.d.nsa, p.d.nopd, p.d.dx, opd, w.use_dm != 0);
	if (r) return r;
	GeomEntry& e = gp.e[gp.nentry - 1];
	e.opdadd = w.opdadd.p;
	e.has_poly = w.has_poly;
	memcpy(e.poly, w.poly, sizeof(e.poly));
	return 0;
}
static void set_llt_poly(GeomEntry& e, const WfsState& w) {
	e.has_poly = w.has_lltpoly;
	memcpy(e.poly, w.lltpoly, sizeof(e.poly));
}
// The LLT pupil of one LGS WFS (maos/wfsgrad.c:337-365): direction
// theta - llt_o/hs, shift llt_o - v*dt*isim, cone of the star, wrap; the
// block then forms the uplink OTF.
static int add_llt_entry(shwfs_ctx* ctx, GeomParams& gp, WfsState& w, int isim) {
	PowfsState& p = ctx->powfs[w.d.ipowfs];
	int r = add_geom_entry(ctx, gp, w.d.thetax - p.d.llt_ox / w.d.hs, w.d.thetay - p.d.llt_oy / w.d.hs, w.d.hs, 0, 0,
		0, p.d.llt_ox, p.d.llt_oy, isim, p.lltorig.p, p.lltorig.p + 1, 1, p.d.llt_nx, p.d.dx, w.lltopd.p);
	if (r) return r;
	GeomEntry& e = gp.e[gp.nentry - 1];
	set_llt_poly(e, w);
	if (p.d.notf != 32) return 0;  // the uplink OTF follows from the traced OPD (launch_uplink_gen)
	e.lltamp = p.lltamp.p;
	e.lotfT = w.lotfT.p;
	e.twoinvwvl = (float)(2.0 / p.d.wvl);
	e.lltnorm = (float)(1.0 / ((double)p.d.llt_nx * p.d.embfac * p.d.llt_nx * p.d.embfac));
	return 0;
}

// The LLT pupil of WFS w once more for wavelength band pb: the uplink OTF at
// the band's wavelength into lotf (the traced OPD is that of the main band's entry).
static int add_llt_band_entry(shwfs_ctx* ctx, GeomParams& gp, WfsState& w, int isim, const PowfsState& pb, float2* lotf) {
	PowfsState& p = ctx->powfs[w.d.ipowfs];
	int r = add_geom_entry(ctx, gp, w.d.thetax - p.d.llt_ox / w.d.hs, w.d.thetay - p.d.llt_oy / w.d.hs, w.d.hs, 0, 0,
		0, p.d.llt_ox, p.d.llt_oy, isim, p.lltorig.p, p.lltorig.p + 1, 1, p.d.llt_nx, p.d.dx, nullptr);
	if (r) return r;
	GeomEntry& e = gp.e[gp.nentry - 1];
	set_llt_poly(e, w);
	e.lltamp = pb.lltamp.p;
	e.lotfT = lotf;
	e.twoinvwvl = (float)(2.0 / pb.d.wvl);
	e.lltnorm = (float)(1.0 / ((double)pb.d.llt_nx * pb.d.embfac * pb.d.llt_nx * pb.d.embfac));
	return 0;
}

static float norm_ints(const PowfsState& p, const WfsState& w) {
	const double nwvf = (double)p.d.nopd * p.d.embfac;
	const double norm_psf = sqrt(p.d.areascale) / ((double)p.d.nopd * nwvf);
	const double wt = p.band_of >= 0 ? p.band_wvlwt : w.d.wvlwt;  // powfs.wvlwts[iwvl]
	return (float)(w.d.sigsim * wt * norm_psf * norm_psf / ((double)p.d.notf * p.d.notf));
}

static PowfsDev make_powfs_dev(const PowfsState& p, int isim) {
	PowfsDev P;
	memset(&P, 0, sizeof(P));
	P.nsa = p.d.nsa;
	P.pixpsax = p.d.pixpsax;
	P.pixpsay = p.d.pixpsay;
	P.npix = p.d.pixpsax * p.d.pixpsay;
	P.etfT1 = p.d.has_etf ? p.etfT[0].p : nullptr;
	// ETF time interpolation (maos/wfsints.c:215-223, cuda/sim/wfsints.cu:362-370)
	P.etfT2 = (p.d.has_etf && p.etfT[1].p && p.etf_dtrat > 0) ? p.etfT[1].p : nullptr;
	P.etfwt1 = 1.f;
	P.etfwt2 = 0.f;
	if (P.etfT2) {
		const double wt2 = (double)(isim % p.etf_dtrat) / (double)p.etf_dtrat;
		P.etfwt2 = (float)wt2;
		P.etfwt1 = (float)(1. - wt2);
	}
	P.nominalT = p.d.has_etf ? nullptr : p.nominalT.p;
	P.nominal_per_sa = p.nnominal > 1;
	P.simap_idx = p.simap_idx.p;
	P.simap_wt = p.simap_wt.p;
	P.simap_per_sa = p.nsimap > 1;
	P.gradtype = p.d.gradtype;
	P.sigmatch = p.d.sigmatch;
	P.cogthres = (float)p.d.cogthres;
	P.cogoff = (float)p.d.cogoff;
	P.pixthetax = (float)p.d.pixthetax;
	P.pixthetay = (float)p.d.pixthetay;
	P.saat = (float)p.d.saat;
	P.sigtot = (float)p.d.sigtot_cog;
	P.saa = p.saa.p;
	P.twoinvwvl = (float)(2.0 / p.d.wvl);
	P.rne = (float)p.d.rne;
	P.bkgrnd = (float)p.d.bkgrnd;
	P.bkgrndc = (float)p.d.bkgrndc;
	P.isim = isim;
	P.lltnorm = (float)(1.0 / ((double)p.d.llt_nx * p.d.embfac * p.d.llt_nx * p.d.embfac));
	P.accum = p.dtrat > 1 && isim % p.dtrat != 0;
	return P;
}

static int check_ready(shwfs_ctx* ctx, const PowfsState& p, const WfsState& w) {
	if (!p.amp.p || !p.origx.p) return fail(ctx, SHWFS_ESTATE, "powfs geometry not set");
	if (p.d.gradtype == SHWFS_GRAD_GTILT) {
		const size_t m = p.namp > 1 ? (size_t)w.wfsind : 0;
		if (m >= p.gs0_ptr.size() || !p.gs0_ptr[m].p) return fail(ctx, SHWFS_ESTATE, "G-tilt operator GS0 not set");
	}
	if (is_geom(p.d.gradtype)) return 0;
	if (!p.simap_idx.p) return fail(ctx, SHWFS_ESTATE, "pixel sampling map not set");
	if (p.d.has_etf && !p.etfT[0].p) return fail(ctx, SHWFS_ESTATE, "ETF not set");
	if (!p.d.has_etf && !p.nominalT.p) return fail(ctx, SHWFS_ESTATE, "DTF nominal not set");
	if (p.d.has_llt && !p.lltamp.p) return fail(ctx, SHWFS_ESTATE, "LLT amplitude not set");
	if (p.d.gradtype == SHWFS_GRAD_MF && !w.mtche.p) return fail(ctx, SHWFS_ESTATE, "matched filter not set");
	if (p.d.gradtype == SHWFS_GRAD_MF && p.d.sigmatch == 1 && !w.i0sum.p) return fail(ctx, SHWFS_ESTATE, "i0sum not set");
	if (p.d.gradtype == SHWFS_GRAD_MF && p.d.sigmatch == 2 && !(w.i0sumsum > 0))
		return fail(ctx, SHWFS_ESTATE, "sigmatch 2: i0sumsum not set");
	return 0;
}

// ---- tensor-core form tables ----
// float -> bf16, round to nearest even
static uint16_t f2bf(float f) {
	uint32_t u;
	memcpy(&u, &f, 4);
	if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;
	u += 0x7fffu + ((u >> 16) & 1u);
	return (uint16_t)(u >> 16);
}
static float bf2f(uint16_t h) {
	uint32_t u = (uint32_t)h << 16;
	float f;
	memcpy(&f, &u, 4);
	return f;
}
// Writes the hi/lo image of a real N x K matrix m(n, k) into the canonical
// K-major layout with 2K/8 chunks per row group (hi chunks first).
static void put_bmat(std::vector<uint16_t>& img, size_t byte0, int N, int K, const std::vector<double>& m) {
	const int kc = 2 * K / 8;
	for (int n = 0; n < N; n++)
		for (int k = 0; k < K; k++) {
			const float v = (float)m[(size_t)n * K + k];
			const uint16_t h = f2bf(v);
			const uint16_t l = f2bf(v - bf2f(h));
			const size_t oh = byte0 + tc_off(n, k / 8, kc) + (k % 8) * 2;
			const size_t ol = byte0 + tc_off(n, K / 8 + k / 8, kc) + (k % 8) * 2;
			img[oh / 2] = h;
			img[ol / 2] = l;
		}
}
// Real block form of a complex matrix M (nout x nin) for C = A B^T with A rows
// [re | im] of length 2*nin: rows n < nout give Re, rows nhalf+n give Im.
static void complex_block(std::vector<double>& m, int N, int K, int nhalf, int nout, int nin,
	const std::vector<double>& mr, const std::vector<double>& mi) {
	m.assign((size_t)N * K, 0.0);
	for (int n = 0; n < nout; n++)
		for (int j = 0; j < nin; j++) {
			const double a = mr[(size_t)n * nin + j], b = mi[(size_t)n * nin + j];
			m[(size_t)n * K + j] = a;
			m[(size_t)n * K + nin + j] = -b;
			m[(size_t)(nhalf + n) * K + j] = b;
			m[(size_t)(nhalf + n) * K + nin + j] = a;
		}
}

// Builds B1 (16-into-32 DFT), B2 (32-point DFT), B3 (Gy) and B4 (Gx) for a powfs.
// The pixel weights come from the pixel geometry in separable form and must
// reproduce the uploaded pixel map tap for tap.
static int build_tc_tables(shwfs_ctx* ctx, PowfsState& p) {
	const shwfs_powfs_desc& d = p.d;
	const int n = d.notf, n2 = n / 2, npx = d.pixpsax, npy = d.pixpsay, npix = npx * npy;
	if (!(d.nopd == 16 && n == 32)) return fail(ctx, SHWFS_EINVAL, "TC form: needs 16x16 OPD points and a 32x32 OTF");
	if (npx > 8 || npy > 8) return fail(ctx, SHWFS_EINVAL, "TC form: at most 8x8 pixels in this build");
	if (p.nsimap != 1 || p.simap_idx_h.empty()) return fail(ctx, SHWFS_EINVAL, "TC form: needs one pixel map shared by all subapertures");
	const double dtheta = d.wvl / (d.dsa * d.embfac);
	const double dx_in1 = 1. / dtheta, disp = (0 - (-n2 * dtheta)) * dx_in1;
	// 1-D bilinear taps of every pixel column / row (lib/mkh.c:96-140 in separable form)
	auto taps = [&](int np, double pth, int i, int* g, double* w) {
		const double po = -(np * 0.5 - 0.5) * pth;
		double f = (i * pth + po) * dx_in1 + disp;
		const int fl = (int)floor(f);
		f -= fl;
		g[0] = fl;
		g[1] = fl + 1;
		w[0] = 1. - f;
		w[1] = f;
	};
	std::vector<double> Wx((size_t)npx * n, 0.0), Wy((size_t)npy * n, 0.0);
	for (int ix = 0; ix < npx; ix++) {
		int g[2];
		double w[2];
		taps(npx, d.pixthetax, ix, g, w);
		for (int iy = 0; iy < npy; iy++) {
			int gy[2];
			double wy[2];
			taps(npy, d.pixthetay, iy, gy, wy);
			// the product taps must equal the uploaded map of pixel (ix, iy)
			std::vector<std::pair<int, double>> mine, theirs;
			for (int b = 0; b < 2; b++)
				for (int a = 0; a < 2; a++) {
					const double wt = w[a] * wy[b];
					if (wt > 1e-15 && g[a] >= 0 && g[a] < n && gy[b] >= 0 && gy[b] < n) mine.push_back({g[a] + gy[b] * n, wt});
				}
			const int pix = ix + iy * npx;
			for (int c = 0; c < 4; c++)
				if (p.simap_idx_h[4 * pix + c] >= 0) theirs.push_back({p.simap_idx_h[4 * pix + c], p.simap_wt_h[4 * pix + c]});
			std::sort(mine.begin(), mine.end());
			std::sort(theirs.begin(), theirs.end());
			bool same = mine.size() == theirs.size();
			for (size_t t = 0; same && t < mine.size(); t++)
				same = mine[t].first == theirs[t].first && fabs(mine[t].second - theirs[t].second) <= 1e-9;
			if (!same) return fail(ctx, SHWFS_EINVAL, "TC form: the pixel map of pixel %d is not separable bilinear", pix);
		}
		for (int a = 0; a < 2; a++)
			if (g[a] >= 0 && g[a] < n) Wx[(size_t)ix * n + g[a]] += w[a];
	}
	for (int iy = 0; iy < npy; iy++) {
		int g[2];
		double w[2];
		taps(npy, d.pixthetay, iy, g, w);
		for (int a = 0; a < 2; a++)
			if (g[a] >= 0 && g[a] < n) Wy[(size_t)iy * n + g[a]] += w[a];
	}
	// G(i, f) = sum_x W(i, x) exp(+2 pi i f x / n)
	auto Gmat = [&](const std::vector<double>& W, int ni, std::vector<double>& gr, std::vector<double>& gi) {
		gr.assign((size_t)ni * n, 0.0);
		gi.assign((size_t)ni * n, 0.0);
		for (int i = 0; i < ni; i++)
			for (int f = 0; f < n; f++)
				for (int x = 0; x < n; x++) {
					const double w = W[(size_t)i * n + x];
					if (w == 0) continue;
					const double ang = 2 * M_PI * (double)((f * x) % n) / n;
					gr[(size_t)i * n + f] += w * cos(ang);
					gi[(size_t)i * n + f] += w * sin(ang);
				}
	};
	std::vector<double> gxr, gxi, gyr, gyi;
	Gmat(Wx, npx, gxr, gxi);
	Gmat(Wy, npy, gyr, gyi);
	// forward DFT matrices, w = exp(-2 pi i / 32)
	std::vector<double> m1r(32 * 16), m1i(32 * 16), m2r(32 * 32), m2i(32 * 32);
	for (int k = 0; k < 32; k++) {
		for (int j = 0; j < 16; j++) {
			const int e = (k * (j + 8)) % 32;
			m1r[k * 16 + j] = cos(2 * M_PI * e / 32);
			m1i[k * 16 + j] = -sin(2 * M_PI * e / 32);
		}
		for (int j = 0; j < 32; j++) {
			const int e = (k * j) % 32;
			m2r[k * 32 + j] = cos(2 * M_PI * e / 32);
			m2i[k * 32 + j] = -sin(2 * M_PI * e / 32);
		}
	}
	std::vector<double> b1, b2, b3, b4((size_t)16 * 64, 0.0);
	complex_block(b1, 64, 32, 32, 32, 16, m1r, m1i);
	complex_block(b2, 64, 64, 32, 32, 32, m2r, m2i);
	complex_block(b3, 32, 64, 16, npy, 32, gyr, gyi);
	// 6b: I(ix, iy) = sum_fx Re T(fx, iy) Re Gx(ix, fx) - Im T(fx, iy) Im Gx(ix, fx)
	for (int i = 0; i < npx; i++)
		for (int f = 0; f < 32; f++) {
			b4[(size_t)i * 64 + f] = gxr[(size_t)i * n + f];
			b4[(size_t)i * 64 + 32 + f] = -gxi[(size_t)i * n + f];
		}
	std::vector<uint16_t> img(TC_B_BYTES / 2, 0);
	put_bmat(img, 0, 64, 32, b1);
	put_bmat(img, TC_B1_BYTES, 64, 64, b2);
	put_bmat(img, TC_B1_BYTES + TC_B2_BYTES, 32, 64, b3);
	put_bmat(img, TC_B1_BYTES + TC_B2_BYTES + TC_B3_BYTES, 16, 64, b4);
	int r;
	if ((r = dev_upload(ctx, p.tc_bmat, reinterpret_cast<const uint4*>(img.data()), TC_B_BYTES / 16))) return r;
	(void)npix;
	p.tc_ready = 1;
	return 0;
}

static int sm_count(shwfs_ctx* ctx) {
	static int nsm[64] = {0};
	if (ctx->device < 64 && nsm[ctx->device]) return nsm[ctx->device];
	int v = 148;
	cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, ctx->device);
	if (ctx->device < 64) nsm[ctx->device] = v;
	return v;
}

// Per-launch WFS descriptors live in a device ring so that queued launches
// never see them overwritten.
static int sync_all_streams(shwfs_ctx* ctx) {
	CK(cudaStreamSynchronize(ctx->stream));
	if (ctx->aux) CK(cudaStreamSynchronize(ctx->aux));
	for (cudaStream_t s : ctx->pstream) CK(cudaStreamSynchronize(s));
	return 0;
}
static const size_t DESC_CACHE_MAX = 64;

static int push_wfsdev(shwfs_ctx* ctx, const std::vector<WfsDev>& wd, const WfsDev** out) {
	const size_t nw = wd.size();
	if (ctx->cache_desc) {
		for (auto& c : ctx->desc_cache)
			if (c.h.size() == nw && !memcmp(c.h.data(), wd.data(), sizeof(WfsDev) * nw)) {
				*out = c.d.p;
				return 0;
			}
		if (ctx->capturing) return fail(ctx, SHWFS_ESTATE, "frame graph: descriptors changed since the warm-up frame");
		if (ctx->desc_cache.size() < DESC_CACHE_MAX) {
			ctx->desc_cache.emplace_back();
			auto& c = ctx->desc_cache.back();
			c.h = wd;
			int r = dev_upload(ctx, c.d, wd.data(), nw);
			if (r) return r;
			*out = c.d.p;
			return 0;
		}
	}
	if (ctx->capturing) return fail(ctx, SHWFS_ESTATE, "frame graph: no cached descriptors");
	const size_t need = ctx->wfsdev_h.size() + nw;
	if (ctx->wfsdev.n < need) {
		if (int r = sync_all_streams(ctx)) return r;
		ctx->wfsdev_h.clear();
		int r = dev_alloc(ctx, ctx->wfsdev, need < 4096 ? 4096 : need * 2);
		if (r) return r;
	}
	if (ctx->wfsdev_h.size() + nw > ctx->wfsdev.n) {
		if (int r = sync_all_streams(ctx)) return r;
		ctx->wfsdev_h.clear();
	}
	const size_t off = ctx->wfsdev_h.size();
	ctx->wfsdev_h.insert(ctx->wfsdev_h.end(), wd.begin(), wd.end());
	CK(cudaMemcpyAsync(ctx->wfsdev.p + off, wd.data(), sizeof(WfsDev) * nw, cudaMemcpyHostToDevice, ctx->stream));
	ctx->h2d_bytes += sizeof(WfsDev) * nw;
	*out = ctx->wfsdev.p + off;
	return 0;
}

// The generic-size chain (n_f = n_w = N in {64, 128, 256}): FFT passes over
// the scratch buf (nitem N^2), WFS or uplink mode.
template <int N>
static int launch_gen_n(shwfs_ctx* ctx, PowfsState& p, GenParams& G) {
	constexpr int L = gen_lines(N);
	const size_t smem = ((size_t)L * (N + 1) + N / 2) * sizeof(float2);
	const dim3 full(G.nitem, N / L), field(G.nitem, (G.nopd + L - 1) / L);
	gen_pass_kernel<N, GEN_FIELD_COLS><<<field, GEN_THREADS, smem, ctx->stream>>>(G);
	gen_pass_kernel<N, GEN_PSF_ROWS><<<full, GEN_THREADS, smem, ctx->stream>>>(G);
	gen_pass_kernel<N, GEN_OTF_COLS><<<full, GEN_THREADS, smem, ctx->stream>>>(G);  // uplink mode: ends at the OTF
	if (!G.uplink) gen_pass_kernel<N, GEN_INV_ROWS><<<full, GEN_THREADS, smem, ctx->stream>>>(G);
	CK(cudaGetLastError());
	(void)p;
	return 0;
}

// twiddles exp(-2 pi i k / N), k < N, of a generic-size powfs
static int ensure_twiddles(shwfs_ctx* ctx, PowfsState& p) {
	if (p.gen_tw.p) return 0;
	const int N = p.d.notf;
	std::vector<float2> tw(N);  // the passes use the first N/2, the fused 64-point kernel all N
	for (int k = 0; k < N; k++) tw[k] = make_float2((float)cos(2 * M_PI * k / N), (float)-sin(2 * M_PI * k / N));
	return dev_upload(ctx, p.gen_tw, tw.data(), tw.size());
}

static int launch_gen(shwfs_ctx* ctx, PowfsState& p, const WfsDev* wdev, int nw, int nitem, int uplink,
	DevBuf<float2>& buf, const PowfsDev& P) {
	const int N = p.d.notf;
	int r;
	if ((r = ensure_twiddles(ctx, p))) return r;
	if (buf.n < (size_t)nitem * N * N) {
		CK(cudaStreamSynchronize(ctx->stream));
		if ((r = dev_alloc(ctx, buf, (size_t)nitem * N * N))) return r;
	}
	GenParams G;
	memset(&G, 0, sizeof(G));
	G.nitem = nitem;
	G.nw = nw;
	G.nopd = uplink ? p.d.llt_nx : p.d.nopd;
	G.pad = (N - G.nopd) / 2;
	G.uplink = uplink;
	G.scale = uplink ? (float)(1.0 / ((double)N * N)) : 1.f;
	G.twoinvwvl = (float)(2.0 / p.d.wvl);
	G.buf = buf.p;
	G.tw = p.gen_tw.p;
	G.wfs = wdev;
	if (!uplink) {
		G.etfT1 = P.etfT1;
		G.etfT2 = P.etfT2;
		G.etfwt1 = P.etfwt1;
		G.etfwt2 = P.etfwt2;
		G.nominalT = P.nominalT;
		G.nominal_per_sa = P.nominal_per_sa;
	}
	switch (N) {
	case 64: return launch_gen_n<64>(ctx, p, G);
	case 128: return launch_gen_n<128>(ctx, p, G);
	case 256: return launch_gen_n<256>(ctx, p, G);
	default: return fail(ctx, SHWFS_EINVAL, "no imaging path for n_f = %d", N);
	}
}

// Uplink OTFs of the LLT pupils of a generic-size powfs from their traced
// OPDs (maos/wfsints.c:149-199).
static int launch_uplink_gen(shwfs_ctx* ctx, PowfsState& p, const std::vector<int>& wlist,
	const std::vector<const float*>& lltopd, const std::vector<float2*>* out = nullptr) {
	std::vector<WfsDev> wd(wlist.size());
	for (size_t k = 0; k < wlist.size(); k++) {
		memset(&wd[k], 0, sizeof(WfsDev));
		wd[k].opd = lltopd[k];
		wd[k].amp = p.lltamp.p;
		wd[k].lotfT = out ? (*out)[k] : ctx->wfs[wlist[k]].lotfT.p;
	}
	const WfsDev* wdev = nullptr;
	int r = push_wfsdev(ctx, wd, &wdev);
	if (r) return r;
	PowfsDev P;
	memset(&P, 0, sizeof(P));
	StageMark m(ctx, SHWFS_STAGE_UPLINK);
	return launch_gen(ctx, p, wdev, (int)wlist.size(), (int)wlist.size(), 1, p.gen_lbuf, P);
}

// (b)-(e) for a set of WFS of one powfs sharing the launch.
static int launch_ints_sig2(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy);
static int launch_ints_dtrat(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy);
static int launch_ints_bands(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy);
static int launch_ints(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy) {
	PowfsState& p = ctx->powfs[ipowfs];
	const int nw = (int)wlist.size();
	if (nw == 0) return 0;
	if (is_geom(p.d.gradtype)) return fail(ctx, SHWFS_EINVAL, "geometric sensor: no imaging");
	if (p.dtrat > 1 && !ctx->dtrat_inner)
		return launch_ints_dtrat(ctx, ipowfs, wlist, isim, opds, lotfs, ints, grads, noisy);
	if (p.d.sigmatch == 2 && !ctx->sig2_inner)
		return launch_ints_sig2(ctx, ipowfs, wlist, isim, opds, lotfs, ints, grads, noisy);
	if (!p.bands.empty() && !ctx->band_inner)
		return launch_ints_bands(ctx, ipowfs, wlist, isim, opds, lotfs, ints, grads, noisy);
	if (ctx->form == SHWFS_FORM_TC && nw > TC_MAX_WFS) {
		// the tensor-core launch holds at most TC_MAX_WFS WFS descriptors in shared memory
		for (int k0 = 0; k0 < nw; k0 += TC_MAX_WFS) {
			const int k1 = std::min(nw, k0 + TC_MAX_WFS);
			auto cut = [&](const auto& v) { return std::vector<typename std::decay_t<decltype(v)>::value_type>(v.begin() + k0, v.begin() + k1); };
			int r = launch_ints(ctx, ipowfs, cut(wlist), isim, cut(opds), cut(lotfs), cut(ints), cut(grads), cut(noisy));
			if (r) return r;
		}
		return 0;
	}
	PowfsDev P = make_powfs_dev(p, isim);
	if (ctx->band_accum) P.accum = 1;
	std::vector<WfsDev> wd(nw);
	for (int k = 0; k < nw; k++) {
		WfsState& w = ctx->wfs[wlist[k]];
		int r = check_ready(ctx, p, w);
		if (r) return r;
		WfsDev& d = wd[k];
		d.opd = opds[k];
		d.amp = p.amp.p + (p.namp > 1 ? (size_t)w.wfsind * p.d.nsa * p.d.nopd * p.d.nopd : 0);
		d.lotfT = lotfs[k];
		d.mtche = w.mtche.p;
		d.i0sum = w.i0sum.p;
		d.ints = ints[k];
		// the tensor-core form passes intensities to its noise/gradient kernel
		if (ctx->form == SHWFS_FORM_TC && !d.ints && grads[k]) {
			if (!w.ints.p) return fail(ctx, SHWFS_ESTATE, "TC form: WFS %d has no intensity buffer", wlist[k]);
			d.ints = w.ints.p;
		}
		d.grad = grads[k];
		d.alpha = norm_ints(p, w);
		d.noisy = noisy[k];
		d.wfs_id = (uint32_t)wlist[k];
		d.seed = w.seed;
	}
	const WfsDev* wdev = nullptr;
	{
		int r = push_wfsdev(ctx, wd, &wdev);
		if (r) return r;
	}
	const int nitem = p.d.nsa * nw;
	const int nblk = (nitem + 3) / 4;
	const int npix = P.npix;
	if (p.d.notf == 64 && npix <= 256) {  // fused per image
		int r = ensure_twiddles(ctx, p);
		if (r) return r;
		StageMark mark(ctx, SHWFS_STAGE_INTS);
		auto kern = p.d.nopd == 32 ? ints_n64_kernel<32> : ints_n64_kernel<0>;
		kern<<<nitem, N64_THREADS, N64_SMEM_BYTES, ctx->stream>>>(P, wdev, nw, nitem, p.d.nopd, (float)(2.0 / p.d.wvl),
			p.gen_tw.p);
		CK(cudaGetLastError());
		return 0;
	}
	if (p.d.notf != 32) {  // generic sizes: FFT passes, then pixels, noise and gradients
		StageMark mark(ctx, SHWFS_STAGE_INTS);
		int r = launch_gen(ctx, p, wdev, nw, nitem, 0, p.gen_buf, P);
		if (r) return r;
		const int n2 = p.d.notf * p.d.notf;
		// a thread per pixel (at most GEN_PIX_THREADS: powfs_add limits these sizes to 256 pixels)
		const int bt = (npix + 31) / 32 * 32;
		gen_pixels_block_kernel<<<nitem, bt, 0, ctx->stream>>>(P, wdev, nw, p.gen_buf.p, n2);
		CK(cudaGetLastError());
		return 0;
	}
	if (ctx->form == SHWFS_FORM_TC) {
		if (!p.tc_ready) {
			int r = build_tc_tables(ctx, p);
			if (r) return r;
		}
		if (!ctx->errflag.p) {
			int r = dev_alloc(ctx, ctx->errflag, 1);
			if (r) return r;
			CK(cudaMemsetAsync(ctx->errflag.p, 0, sizeof(int), ctx->stream));
		}
		static bool attr_set[64] = {false};
		if (ctx->device < 64 && !attr_set[ctx->device]) {
			CK(cudaFuncSetAttribute(ints_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
				tc_smem_bytes(TC_MAX_WFS)));
			attr_set[ctx->device] = true;
		}
		TcTables T{p.tc_bmat.p};
		bool all_lotf = true, any_out = false;
		for (int k = 0; k < nw; k++) {
			all_lotf = all_lotf && wd[k].lotfT;
			any_out = any_out || wd[k].ints;
		}
		const int nlotf = all_lotf ? nw : 0;
		// persistent: TC_CTAS_PER_SM CTAs of TC_GROUPS tile groups per SM
		const int ntile = (nitem + 3) / 4;
		const int grid = std::min((ntile + TC_GROUPS - 1) / TC_GROUPS, sm_count(ctx) * TC_CTAS_PER_SM);
		if (any_out) {
			StageMark mark(ctx, SHWFS_STAGE_INTS);
			ints_tc_kernel<<<grid, TC_THREADS, tc_smem_bytes(nlotf), ctx->stream>>>(P, wdev, nw, nitem, nlotf, T,
				ctx->errflag.p);
			ctx->errflag_armed = 1;
		}
		CK(cudaGetLastError());
		bool post = false;
		for (int k = 0; k < nw; k++) post = post || (wd[k].ints && (wd[k].noisy || wd[k].grad));
		if (post) {
			StageMark mark(ctx, SHWFS_STAGE_POST);
			if (npix <= 32) noise_grad_kernel<1><<<nblk, 128, 0, ctx->stream>>>(P, wdev, nw, nitem);
			else noise_grad_kernel<2><<<nblk, 128, 0, ctx->stream>>>(P, wdev, nw, nitem);
			CK(cudaGetLastError());
		}
		return 0;
	}
	StageMark mark(ctx, SHWFS_STAGE_INTS);
	const int v = p.band_of >= 0 ? ctx->powfs[p.band_of].variant : p.variant;  // a band follows its main powfs
	auto go = [&](auto kern) { kern<<<nblk, 128, 0, ctx->stream>>>(P, wdev, nw, nitem); };
	// variants 0-2: full-spectrum transforms at a register cap for 4, 5, 6
	// blocks per SM; 3-5: the half-spectrum form at the same caps
	if (npix <= 32) {
		if (v == 1) go(ints_n32_kernel<1, 5>);
		else if (v == 2) go(ints_n32_kernel<1, 6>);
		else if (v == 3) go(ints_n32_kernel<1, 4, true>);
		else if (v == 4) go(ints_n32_kernel<1, 5, true>);
		else if (v == 5) go(ints_n32_kernel<1, 6, true>);
		else go(ints_n32_kernel<1, 4>);
	} else if (npix <= 64) {
		if (v == 1) go(ints_n32_kernel<2, 5>);
		else if (v == 2) go(ints_n32_kernel<2, 6>);
		else if (v == 3) go(ints_n32_kernel<2, 4, true>);
		else if (v == 4) go(ints_n32_kernel<2, 5, true>);
		else if (v == 5) go(ints_n32_kernel<2, 6, true>);
		else go(ints_n32_kernel<2, 4>);
	} else {
		if (v == 1) go(ints_n32_kernel<4, 5>);
		else if (v == 2) go(ints_n32_kernel<4, 6>);
		else if (v == 3) go(ints_n32_kernel<4, 4, true>);
		else if (v == 4) go(ints_n32_kernel<4, 5, true>);
		else if (v == 5) go(ints_n32_kernel<4, 6, true>);
		else go(ints_n32_kernel<4, 4>);
	}
	CK(cudaGetLastError());
	return 0;
}

static int launch_uplink(shwfs_ctx* ctx, const std::vector<int>& wlist, const std::vector<const float*>& lltopd,
	std::vector<const float2*>& lotfs) {
	if (wlist.empty()) return 0;
	PowfsState& p = ctx->powfs[ctx->wfs[wlist[0]].d.ipowfs];
	const int nw = (int)wlist.size();
	if (p.d.notf != 32) {
		for (int k = 0; k < nw; k++) lotfs[k] = ctx->wfs[wlist[k]].lotfT.p;
		return launch_uplink_gen(ctx, p, wlist, lltopd);
	}
	std::vector<const float*> in(nw);
	std::vector<float2*> out(nw);
	for (int k = 0; k < nw; k++) {
		in[k] = lltopd[k];
		out[k] = ctx->wfs[wlist[k]].lotfT.p;
		lotfs[k] = out[k];
	}
	CK(cudaStreamSynchronize(ctx->stream));
	int r;
	if ((r = dev_alloc(ctx, ctx->llt_in, (size_t)nw))) return r;
	if ((r = dev_alloc(ctx, ctx->llt_out, (size_t)nw))) return r;
	CK(cudaMemcpyAsync(ctx->llt_in.p, in.data(), sizeof(float*) * nw, cudaMemcpyHostToDevice, ctx->stream));
	CK(cudaMemcpyAsync(ctx->llt_out.p, out.data(), sizeof(float2*) * nw, cudaMemcpyHostToDevice, ctx->stream));
	ctx->h2d_bytes += (sizeof(float*) + sizeof(float2*)) * nw;
	const float twoinvwvl = (float)(2.0 / p.d.wvl);
	const float lltnorm = (float)(1.0 / ((double)p.d.llt_nx * p.d.embfac * p.d.llt_nx * p.d.embfac));
	{
		StageMark m(ctx, SHWFS_STAGE_UPLINK);
		uplink_otf_n32_kernel<<<(nw + 3) / 4, 128, 0, ctx->stream>>>(ctx->llt_in.p, p.lltamp.p, ctx->llt_out.p, nw,
			twoinvwvl, lltnorm);
	}
	CK(cudaGetLastError());
	return 0;
}

// Imaging of a powfs that integrates dtrat frames per output frame
// (powfs.dtrat, maos/wfsgrad.c: intensities accumulate in wfsints and noise
// and gradients are formed on the frame with (isim + 1) % dtrat == 0): each
// WFS's intensity buffer holds the sum; the first frame of a period starts
// it, the others add to it, and the last adds noise and forms the gradients.
static int launch_ints_dtrat(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy) {
	PowfsState& p = ctx->powfs[ipowfs];
	const int nw = (int)wlist.size();
	if (isim < 0) return fail(ctx, SHWFS_EINVAL, "dtrat: negative frame index");
	const bool out = (isim + 1) % p.dtrat == 0;
	std::vector<float*> acc(nw), gr(nw, nullptr);
	std::vector<int> nz(nw, 0);
	for (int k = 0; k < nw; k++) {
		WfsState& w = ctx->wfs[wlist[k]];
		if (!w.ints.p) return fail(ctx, SHWFS_ESTATE, "dtrat: WFS %d has no intensity buffer", wlist[k]);
		acc[k] = w.ints.p;
		if (out) {
			gr[k] = grads[k];
			nz[k] = noisy[k];
		}
	}
	ctx->dtrat_inner = 1;
	int r = launch_ints(ctx, ipowfs, wlist, isim, opds, lotfs, acc, gr, nz);
	ctx->dtrat_inner = 0;
	if (r) return r;
	if (out)
		for (int k = 0; k < nw; k++)
			if (ints[k] && ints[k] != acc[k])
				CK(cudaMemcpyAsync(ints[k], acc[k], sizeof(float) * p.d.nsa * p.d.pixpsax * p.d.pixpsay,
					cudaMemcpyDeviceToDevice, ctx->stream));
	return 0;
}

// Imaging of a powfs with wavelength bands (maos/wfsints.c:145-288, the loop
// over powfs.wvl): every band images the same OPD with its own wavelength,
// uplink OTF, transfer function and pixel map, and adds its intensities, times
// its weight, to those of the bands before it; noise and gradients follow on
// the sum, in the launch of the last band.
static int launch_ints_bands(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy) {
	const int nw = (int)wlist.size();
	std::vector<int> order(1, ipowfs);
	for (int b : ctx->powfs[ipowfs].bands) order.push_back(b);
	std::vector<float*> acc(nw), none(nw, nullptr);
	std::vector<int> quiet(nw, 0);
	for (int k = 0; k < nw; k++) {
		acc[k] = ints[k] ? ints[k] : ctx->wfs[wlist[k]].ints.p;
		if (!acc[k]) return fail(ctx, SHWFS_ESTATE, "bands: WFS %d has no intensity buffer", wlist[k]);
	}
	const int accum0 = ctx->band_accum;
	int r = 0;
	ctx->band_inner = 1;
	for (size_t j = 0; j < order.size() && !r; j++) {
		const bool last = j + 1 == order.size();
		std::vector<const float2*> lj(nw, nullptr);
		for (int k = 0; k < nw; k++) {
			if (j == 0) {
				lj[k] = lotfs[k];
			} else if (ctx->powfs[order[j]].d.has_llt) {
				const auto& bl = ctx->powfs[order[j]].band_lotf;
				if ((size_t)wlist[k] >= bl.size() || !bl[wlist[k]].p) {
					r = fail(ctx, SHWFS_ESTATE, "bands: the uplink OTF of WFS %d is formed by the frame path", wlist[k]);
					break;
				}
				lj[k] = bl[wlist[k]].p;
			}
		}
		if (r) break;
		ctx->band_accum = j > 0 ? 1 : accum0;
		r = launch_ints(ctx, order[j], wlist, isim, opds, lj, acc, last ? grads : none, last ? noisy : quiet);
	}
	ctx->band_inner = 0;
	ctx->band_accum = accum0;
	return r;
}

// Imaging of a sigmatch-2 powfs (normalisation by the frame's total
// intensity, maos/utils.c:1013-1036): intensities with noise first, then the
// total of each WFS (ints_sum_kernel), then the gradients (grad_sig2_kernel).
static int launch_ints_sig2(shwfs_ctx* ctx, int ipowfs, const std::vector<int>& wlist, int isim,
	const std::vector<const float*>& opds, const std::vector<const float2*>& lotfs, const std::vector<float*>& ints,
	const std::vector<float*>& grads, const std::vector<int>& noisy) {
	PowfsState& p = ctx->powfs[ipowfs];
	const int nw = (int)wlist.size();
	std::vector<float*> in(ints), none(nw, nullptr);
	for (int k = 0; k < nw; k++) {
		WfsState& w = ctx->wfs[wlist[k]];
		if (!in[k]) in[k] = w.ints.p;
		if (!in[k]) return fail(ctx, SHWFS_ESTATE, "sigmatch 2: WFS %d has no intensity buffer", wlist[k]);
		int r = dev_alloc(ctx, w.i1sum, 1);
		if (r) return r;
	}
	ctx->sig2_inner = 1;
	int r = launch_ints(ctx, ipowfs, wlist, isim, opds, lotfs, in, none, noisy);
	ctx->sig2_inner = 0;
	if (r) return r;
	const PowfsDev P = make_powfs_dev(p, isim);
	const long n = (long)p.d.nsa * P.npix;
	for (int k0 = 0; k0 < nw; k0 += GEOM_SUM_MAX) {
		SumParams S;
		memset(&S, 0, sizeof(S));
		S.nw = std::min(GEOM_SUM_MAX, nw - k0);
		S.n = n;
		for (int k = 0; k < S.nw; k++) {
			WfsState& w = ctx->wfs[wlist[k0 + k]];
			CK(cudaMemsetAsync(w.i1sum.p, 0, sizeof(double), ctx->stream));
			S.ints[k] = in[k0 + k];
			S.sum[k] = w.i1sum.p;
		}
		const int nblk = (int)std::min((n + 255) / 256, (long)64);
		StageMark m(ctx, SHWFS_STAGE_POST);
		ints_sum_kernel<<<dim3(nblk, S.nw), 256, 0, ctx->stream>>>(S);
		CK(cudaGetLastError());
	}
	for (int k = 0; k < nw; k++) {
		if (!grads[k]) continue;
		WfsState& w = ctx->wfs[wlist[k]];
		const int nblk = (p.d.nsa + 3) / 4;
		StageMark m(ctx, SHWFS_STAGE_POST);
		if (P.npix <= 32)
			grad_sig2_kernel<1><<<nblk, 128, 0, ctx->stream>>>(P, in[k], w.mtche.p, w.i0sum.p, grads[k], w.i1sum.p,
				w.i0sumsum, p.saasum);
		else if (P.npix <= 64)
			grad_sig2_kernel<2><<<nblk, 128, 0, ctx->stream>>>(P, in[k], w.mtche.p, w.i0sum.p, grads[k], w.i1sum.p,
				w.i0sumsum, p.saasum);
		else if (P.npix <= 128)
			grad_sig2_kernel<4><<<nblk, 128, 0, ctx->stream>>>(P, in[k], w.mtche.p, w.i0sum.p, grads[k], w.i1sum.p,
				w.i0sumsum, p.saasum);
		else
			grad_sig2_kernel<8><<<nblk, 128, 0, ctx->stream>>>(P, in[k], w.mtche.p, w.i0sum.p, grads[k], w.i1sum.p,
				w.i0sumsum, p.saasum);
		CK(cudaGetLastError());
	}
	return 0;
}

extern "C" {

int shwfs_raytrace_dev(shwfs_ctx* ctx, int iwfs, int isim, float* opd) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || !opd) return ctx ? fail(ctx, SHWFS_EINVAL, "raytrace: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	GeomParams gp;
	geom_init(ctx, gp);
	if ((r = add_wfs_entry(ctx, gp, *w, isim, opd))) return r;
	return launch_geom(ctx, gp);
}

int shwfs_ints_grad_dev(shwfs_ctx* ctx, int iwfs, int isim, const float* opd, const float* lltopd, float* ints,
	float* grad, int add_noise) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || !opd) return ctx ? fail(ctx, SHWFS_EINVAL, "ints_grad: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	std::vector<int> wl{iwfs};
	std::vector<const float2*> lotf{nullptr};
	if (p.d.has_llt) {
		if (!lltopd) return fail(ctx, SHWFS_EINVAL, "ints_grad: LGS powfs needs the LLT OPD");
		if (!p.bands.empty())
			return fail(ctx, SHWFS_EINVAL,
				"ints_grad: an LGS powfs with wavelength bands forms its uplink OTFs in the frame path (shwfs_frame_queue)");
		if (!p.lltamp.p) return fail(ctx, SHWFS_ESTATE, "LLT amplitude not set");
		std::vector<const float*> lin{lltopd};
		if ((r = launch_uplink(ctx, wl, lin, lotf))) return r;
	}
	std::vector<const float*> opds{opd};
	std::vector<float*> in{ints}, gr{grad};
	std::vector<int> nz{(add_noise && w->d.noisy) ? 1 : 0};
	return launch_ints(ctx, w->d.ipowfs, wl, isim, opds, lotf, in, gr, nz);
}

int shwfs_grad_dev(shwfs_ctx* ctx, int iwfs, const float* ints, float* grad) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || !ints || !grad) return ctx ? fail(ctx, SHWFS_EINVAL, "grad: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	if (is_geom(p.d.gradtype)) return fail(ctx, SHWFS_EINVAL, "grad: geometric sensor has no pixels");
	if (p.d.gradtype == SHWFS_GRAD_MF && !w->mtche.p) return fail(ctx, SHWFS_ESTATE, "matched filter not set");
	PowfsDev P = make_powfs_dev(p, 0);
	const int nblk = (p.d.nsa + 3) / 4;
	if (p.d.sigmatch == 2) {
		// the total intensity of the given frame first (maos/utils.c:1022-1026)
		if (p.d.gradtype == SHWFS_GRAD_MF && !(w->i0sumsum > 0)) return fail(ctx, SHWFS_ESTATE, "sigmatch 2: i0sumsum not set");
		if ((r = dev_alloc(ctx, w->i1sum, 1))) return r;
		CK(cudaMemsetAsync(w->i1sum.p, 0, sizeof(double), ctx->stream));
		SumParams S;
		memset(&S, 0, sizeof(S));
		S.nw = 1;
		S.n = (long)p.d.nsa * P.npix;
		S.ints[0] = ints;
		S.sum[0] = w->i1sum.p;
		ints_sum_kernel<<<dim3((unsigned)std::min((S.n + 255) / 256, 64L), 1), 256, 0, ctx->stream>>>(S);
		CK(cudaGetLastError());
		if (P.npix <= 32)
			grad_sig2_kernel<1><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad, w->i1sum.p, w->i0sumsum, p.saasum);
		else if (P.npix <= 64)
			grad_sig2_kernel<2><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad, w->i1sum.p, w->i0sumsum, p.saasum);
		else if (P.npix <= 128)
			grad_sig2_kernel<4><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad, w->i1sum.p, w->i0sumsum, p.saasum);
		else
			grad_sig2_kernel<8><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad, w->i1sum.p, w->i0sumsum, p.saasum);
		CK(cudaGetLastError());
		return 0;
	}
	if (P.npix <= 32)
		grad_kernel<1><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad);
	else if (P.npix <= 64)
		grad_kernel<2><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad);
	else
		grad_kernel<4><<<nblk, 128, 0, ctx->stream>>>(P, ints, w->mtche.p, w->i0sum.p, grad);
	CK(cudaGetLastError());
	return 0;
}

int shwfs_addnoise_dev(shwfs_ctx* ctx, float* ints, long n, const float* bkgrnd2, const float* bkgrnd2c,
	const float* qe, double bkgrnd, double bkgrndc, double rne, double excess, uint64_t seed, uint32_t stream,
	uint32_t frame) {
	if (!ctx || n < 0 || (n > 0 && !ints) || n > 0xffffffffL)
		return ctx ? fail(ctx, SHWFS_EINVAL, "addnoise: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (n == 0) return 0;
	if (excess < 1) excess = 1;
	const long nblk = std::min((n + 255) / 256, (long)sm_count(ctx) * 8);
	addnoise_kernel<<<(int)nblk, 256, 0, ctx->stream>>>(ints, n, bkgrnd2, bkgrnd2c, qe, (float)bkgrnd,
		(float)bkgrndc, (float)rne, (float)excess, seed, stream, frame);
	CK(cudaGetLastError());
	return 0;
}

// Geometric gradients of one WFS from its OPD (one warp per subaperture):
// z-tilt, or G-tilt with the WFS's GS0.
static int launch_geom_grad(shwfs_ctx* ctx, WfsState& w, const float* opd, float* grad, bool noisy, int isim) {
	PowfsState& p = ctx->powfs[w.d.ipowfs];
	const int nsa = p.d.nsa;
	const float* nea = noisy ? w.neasim.p : nullptr;
	const uint32_t wid = (uint32_t)(&w - ctx->wfs.data());
	if (p.d.gradtype == SHWFS_GRAD_GTILT) {
		const size_t m = p.namp > 1 ? (size_t)w.wfsind : 0;
		if (m >= p.gs0_ptr.size() || !p.gs0_ptr[m].p) return fail(ctx, SHWFS_ESTATE, "G-tilt operator GS0 not set");
		StageMark mk(ctx, SHWFS_STAGE_POST);
		gtilt_kernel<<<(nsa + 7) / 8, 256, 0, ctx->stream>>>(p.gs0_ptr[m].p, p.gs0_col[m].p, p.gs0_val[m].p, nsa, opd,
			grad, nea, w.seed, wid, (uint32_t)isim);
	} else {
		const float* amp = p.amp.p + (p.namp > 1 ? (size_t)w.wfsind * nsa * p.d.nopd * p.d.nopd : 0);
		StageMark mk(ctx, SHWFS_STAGE_POST);
		ztilt_kernel<<<(nsa + 7) / 8, 256, 0, ctx->stream>>>(opd, amp, p.origx.p, p.origy.p, nsa, p.d.nopd, p.d.dx,
			grad, nea, w.seed, wid, (uint32_t)isim);
	}
	CK(cudaGetLastError());
	return 0;
}

// The work of one powfs in a frame: ray trace (and uplink), then imaging.
static int trace_powfs(shwfs_ctx* ctx, int ip, const std::vector<int>& wl, int isim);
static int frame_powfs(shwfs_ctx* ctx, int ip, const std::vector<int>& wl, int isim) {
	PowfsState& p = ctx->powfs[ip];
	int r;
	if (is_geom(p.d.gradtype)) {
		for (size_t b = 0; b < wl.size(); b += SHWFS_MAX_ENTRIES) {
			GeomParams gp;
			geom_init(ctx, gp);
			for (size_t k = b; k < wl.size() && k < b + SHWFS_MAX_ENTRIES; k++) {
				WfsState& w = ctx->wfs[wl[k]];
				if ((r = add_wfs_entry(ctx, gp, w, isim, w.opd.p))) return r;
			}
			if ((r = launch_geom(ctx, gp))) return r;
		}
		for (int i : wl) {
			WfsState& w = ctx->wfs[i];
			if ((r = launch_geom_grad(ctx, w, w.opd.p, w.grad.p, w.d.noisy && w.neasim.p, isim))) return r;
		}
		return 0;
	}
	if ((r = trace_powfs(ctx, ip, wl, isim))) return r;
	// (b)-(e)
	std::vector<const float*> opds;
	std::vector<const float2*> lotf;
	std::vector<float*> in, gr;
	std::vector<int> nz;
	for (int i : wl) {
		WfsState& w = ctx->wfs[i];
		opds.push_back(w.opd.p);
		lotf.push_back(p.d.has_llt ? w.lotfT.p : nullptr);
		in.push_back(w.ints.p);
		gr.push_back(w.grad.p);
		nz.push_back(w.d.noisy);
	}
	return launch_ints(ctx, ip, wl, isim, opds, lotf, in, gr, nz);
}

// (a) of a physical-optics powfs: one ray-trace launch per batch of pupils
// (WFS + LLT), and the uplink OTFs of the larger sizes.
static int trace_powfs(shwfs_ctx* ctx, int ip, const std::vector<int>& wl, int isim) {
	PowfsState& p = ctx->powfs[ip];
	int r;
	// each wavelength band of an LGS powfs forms its own uplink OTF per WFS
	const int nb = (int)p.bands.size();
	if (p.d.has_llt && nb) {
		for (int ib : p.bands) {
			PowfsState& pb = ctx->powfs[ib];
			if (pb.band_lotf.size() < ctx->wfs.size()) pb.band_lotf.resize(ctx->wfs.size());
			for (int i : wl) {
				if (pb.band_lotf[i].p) continue;
				if (ctx->capturing) return fail(ctx, SHWFS_ESTATE, "frame graph: band buffers not allocated by a warm-up frame");
				if ((r = dev_alloc(ctx, pb.band_lotf[i], (size_t)pb.d.notf * pb.d.notf))) return r;
			}
		}
	}
	const int per = p.d.has_llt ? SHWFS_MAX_ENTRIES / (2 + (p.d.notf == 32 ? nb : 0)) : SHWFS_MAX_ENTRIES;
	for (size_t b = 0; b < wl.size(); b += per) {
		GeomParams gp;
		geom_init(ctx, gp);
		for (size_t k = b; k < wl.size() && k < b + per; k++) {
			WfsState& w = ctx->wfs[wl[k]];
			if ((r = add_wfs_entry(ctx, gp, w, isim, w.opd.p))) return r;
			if (p.d.has_llt && (r = add_llt_entry(ctx, gp, w, isim))) return r;
			if (p.d.has_llt && p.d.notf == 32)
				for (int ib : p.bands)
					if ((r = add_llt_band_entry(ctx, gp, w, isim, ctx->powfs[ib], ctx->powfs[ib].band_lotf[wl[k]].p)))
						return r;
		}
		if ((r = launch_geom(ctx, gp))) return r;
		if (p.d.has_llt && p.d.notf != 32) {
			std::vector<int> bw;
			std::vector<const float*> lo;
			for (size_t k = b; k < wl.size() && k < b + per; k++) {
				bw.push_back(wl[k]);
				lo.push_back(ctx->wfs[wl[k]].lltopd.p);
			}
			if ((r = launch_uplink_gen(ctx, p, bw, lo))) return r;
			for (int ib : p.bands) {
				std::vector<float2*> out;
				for (int i : bw) out.push_back(ctx->powfs[ib].band_lotf[i].p);
				if ((r = launch_uplink_gen(ctx, ctx->powfs[ib], bw, lo, &out))) return r;
			}
		}
	}
	return 0;
}

// The branch of a powfs with fewer images per frame than the largest powfs of
// the context runs at the device's greatest stream priority (captured into the
// frame graph as node priorities): the small sensors' chains of dependent
// launches (the FFT-pass chain of one NGS image) then take SMs as the large
// imaging kernel's blocks retire, instead of queueing behind all of them.
static int ensure_branches(shwfs_ctx* ctx) {
	if (ctx->pstream.size() >= ctx->powfs.size()) return 0;
	std::vector<long> nimg(ctx->powfs.size(), 0);
	for (const WfsState& w : ctx->wfs) nimg[w.d.ipowfs] += ctx->powfs[w.d.ipowfs].d.nsa;
	const long nmax = *std::max_element(nimg.begin(), nimg.end());
	int lo = 0, hi = 0;
	CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
	while (ctx->pstream.size() < ctx->powfs.size()) {
		cudaStream_t st;
		cudaEvent_t a, b;
		const size_t ip = ctx->pstream.size();
		CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking,
			ctx->branch_priority && nimg[ip] < nmax ? hi : std::min(lo, std::max(hi, ctx->priority))));
		CK(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
		CK(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
		ctx->pstream.push_back(st);
		ctx->ev_pfork.push_back(a);
		ctx->ev_pjoin.push_back(b);
	}
	return 0;
}

static bool variant_half(int v) { return v >= 3; }

// The powfs the work-list launch serves: FFT form, physical optics, 32-point
// (at most 128 pixels) or 128/256-point (at most 256 pixels), one frame per
// output frame (dtrat 1), sigmatch 0 or 1.
static bool worklist_serves(const shwfs_ctx* ctx, const PowfsState& p) {
	if (ctx->form != SHWFS_FORM_FFT || is_geom(p.d.gradtype) || p.dtrat > 1 || p.d.sigmatch == 2 || !p.bands.empty())
		return false;
	const int npix = p.d.pixpsax * p.d.pixpsay;
	if (p.d.notf == 32) return p.d.nopd == 16 && npix <= 128;
	return (p.d.notf == 128 || p.d.notf == 256) && npix <= 256;
}

// One frame of the powfs in wl as ray traces, then one persistent imaging
// launch over a work list (worklist_kernel).  Geometric powfs run their own
// chain first.  Returns 1 (nothing queued) when a powfs is not served.
static int frame_worklist(shwfs_ctx* ctx, const std::vector<std::vector<int>>& wl, int isim) {
	int nseg = 0, nhalf = 0, nfull = 0;
	for (size_t ip = 0; ip < wl.size(); ip++) {
		if (wl[ip].empty() || is_geom(ctx->powfs[ip].d.gradtype)) continue;
		if (!worklist_serves(ctx, ctx->powfs[ip])) return 1;
		nseg++;
		if (ctx->powfs[ip].d.notf == 32) (variant_half(ctx->powfs[ip].variant) ? nhalf : nfull)++;
	}
	// one form for the frame's 32-point images: that of their powfs' variants
	if (nhalf && nfull) return 1;
	const bool half32 = nhalf > 0;
	if (nseg == 0 || nseg > WL_MAX_SEG) return 1;
	int r;
	// the ray traces of the powfs (and the whole chain of a geometric one) run
	// side by side: the first on the context stream, the others on the powfs
	// branches, joined before the imaging launch
	int nbr = 0;
	for (size_t ip = 0; ip < wl.size(); ip++) nbr += !wl[ip].empty();
	if (nbr > 1 && !ctx->capturing && (r = ensure_branches(ctx))) return r;
	if (nbr > 1 && ctx->pstream.size() < ctx->powfs.size())
		return fail(ctx, SHWFS_ESTATE, "frame graph: stream branches not created by a warm-up frame");
	cudaStream_t main = ctx->stream;
	bool first = true;
	if (nbr > 1) CK(cudaEventRecord(ctx->ev_pfork[0], main));
	for (size_t ip = 0; ip < wl.size(); ip++) {
		if (wl[ip].empty()) continue;
		const bool branch = nbr > 1 && !first;
		if (branch) {
			CK(cudaStreamWaitEvent(ctx->pstream[ip], ctx->ev_pfork[0], 0));
			ctx->stream = ctx->pstream[ip];
		}
		if (is_geom(ctx->powfs[ip].d.gradtype)) r = frame_powfs(ctx, (int)ip, wl[ip], isim);
		else r = trace_powfs(ctx, (int)ip, wl[ip], isim);
		ctx->stream = main;
		if (branch) {
			CK(cudaEventRecord(ctx->ev_pjoin[ip], ctx->pstream[ip]));
			CK(cudaStreamWaitEvent(main, ctx->ev_pjoin[ip], 0));
		}
		first = false;
		if (r) return r;
	}
	if (!ctx->errflag.p) {
		if ((r = dev_alloc(ctx, ctx->errflag, 1))) return r;
		CK(cudaMemsetAsync(ctx->errflag.p, 0, sizeof(int), ctx->stream));
	}
	WorkParams W;
	memset(&W, 0, sizeof(W));
	int nimg_big = 0;
	std::vector<int4> b_tiles[7], pix, n32;
	for (size_t ip = 0; ip < wl.size(); ip++) {
		if (wl[ip].empty() || is_geom(ctx->powfs[ip].d.gradtype)) continue;
		PowfsState& p = ctx->powfs[ip];
		const int nw = (int)wl[ip].size(), nitem = p.d.nsa * nw, si = W.nseg++;
		WorkSeg& S = W.seg[si];
		S.P = make_powfs_dev(p, isim);
		std::vector<WfsDev> wd(nw);
		for (int k = 0; k < nw; k++) {
			WfsState& w = ctx->wfs[wl[ip][k]];
			WfsDev& d = wd[k];
			memset(&d, 0, sizeof(d));
			d.opd = w.opd.p;
			d.amp = p.amp.p + (p.namp > 1 ? (size_t)w.wfsind * p.d.nsa * p.d.nopd * p.d.nopd : 0);
			d.lotfT = p.d.has_llt ? w.lotfT.p : nullptr;
			d.mtche = w.mtche.p;
			d.i0sum = w.i0sum.p;
			d.ints = w.ints.p;
			d.grad = w.grad.p;
			d.alpha = norm_ints(p, w);
			d.noisy = w.d.noisy;
			d.wfs_id = (uint32_t)wl[ip][k];
			d.seed = w.seed;
		}
		if ((r = push_wfsdev(ctx, wd, &S.wfs))) return r;
		S.nw = nw;
		S.nitem = nitem;
		S.n = p.d.notf;
		const int npix = p.d.pixpsax * p.d.pixpsay;
		S.npq = npix <= 32 ? 1 : npix <= 64 ? 2 : npix <= 128 ? 4 : 8;
		if (S.n == 32) {
			const int g = std::max(1, ctx->wl_group);
			for (int a = 0; a < nitem; a += g) n32.push_back(make_int4(WL_N32, si, a, g));
			continue;
		}
		// the pass chain of the large images, as launch_gen sets it up
		const int N = S.n;
		if ((r = ensure_twiddles(ctx, p))) return r;
		if (p.gen_buf.n < (size_t)nitem * N * N) {
			if (ctx->capturing) return fail(ctx, SHWFS_ESTATE, "frame graph: scratch not allocated by a warm-up frame");
			CK(cudaStreamSynchronize(ctx->stream));
			if ((r = dev_alloc(ctx, p.gen_buf, (size_t)nitem * N * N))) return r;
		}
		GenParams& G = S.G;
		G.nitem = nitem;
		G.nw = nw;
		G.nopd = p.d.nopd;
		G.pad = (N - G.nopd) / 2;
		G.uplink = 0;
		G.scale = 1.f;
		G.twoinvwvl = (float)(2.0 / p.d.wvl);
		G.buf = p.gen_buf.p;
		G.tw = p.gen_tw.p;
		G.wfs = S.wfs;
		G.etfT1 = S.P.etfT1;
		G.etfT2 = S.P.etfT2;
		G.etfwt1 = S.P.etfwt1;
		G.etfwt2 = S.P.etfwt2;
		G.nominalT = S.P.nominalT;
		G.nominal_per_sa = S.P.nominal_per_sa;
		const int L = gen_lines(N);
		S.nt1 = (G.nopd + L - 1) / L;
		S.ntf = N / L;
		S.img0 = nimg_big;
		nimg_big += nitem;
		for (int i = 0; i < nitem; i++) {
			for (int t = 0; t < S.nt1; t++) b_tiles[1].push_back(make_int4(WL_TILE, si, i, (1 << 16) | t));
			for (int ps = 2; ps <= GEN_NPASS; ps++)
				for (int t = 0; t < S.ntf; t++) b_tiles[ps].push_back(make_int4(WL_TILE, si, i, (ps << 16) | t));
		}
		for (int a = 0; a < nitem; a += 4) pix.push_back(make_int4(WL_PIX, si, a, 0));
	}
	// the list: pass 1 tiles, a slice of 32-point groups, pass 2 tiles, a slice, ...,
	// the last pass's tiles, a slice, the large images' pixels, the rest of the 32-point groups
	std::vector<int4> list;
	const int ns = std::max(GEN_NPASS + 1, ctx->wl_slices);
	const size_t per = (n32.size() + ns - 1) / ns;
	size_t k = 0;
	for (int ps = 1; ps <= GEN_NPASS; ps++) {
		list.insert(list.end(), b_tiles[ps].begin(), b_tiles[ps].end());
		for (size_t e = std::min(n32.size(), k + per); k < e; k++) list.push_back(n32[k]);
	}
	list.insert(list.end(), pix.begin(), pix.end());
	for (; k < n32.size(); k++) list.push_back(n32[k]);
	// the list repeats from frame to frame: kept on the device
	const int4* dlist = nullptr;
	for (auto& c : ctx->wl_cache)
		if (c.h.size() == list.size() && !memcmp(c.h.data(), list.data(), sizeof(int4) * list.size())) dlist = c.d.p;
	if (!dlist) {
		if (ctx->capturing) return fail(ctx, SHWFS_ESTATE, "frame graph: work list changed since the warm-up frame");
		if (ctx->wl_cache.size() >= 8) {
			CK(cudaStreamSynchronize(ctx->stream));
			for (auto& c : ctx->wl_cache) c.d.free_();
			ctx->wl_cache.clear();
		}
		ctx->wl_cache.emplace_back();
		auto& c = ctx->wl_cache.back();
		c.h = list;
		if ((r = dev_upload(ctx, c.d, list.data(), list.size()))) return r;
		dlist = c.d.p;
	}
	const size_t ncnt = 1 + (size_t)nimg_big;
	if (ctx->wl_cnt.n < ncnt) {
		if (ctx->capturing) return fail(ctx, SHWFS_ESTATE, "frame graph: counters not allocated by a warm-up frame");
		CK(cudaStreamSynchronize(ctx->stream));
		if ((r = dev_alloc(ctx, ctx->wl_cnt, std::max(ncnt, (size_t)64)))) return r;
	}
	CK(cudaMemsetAsync(ctx->wl_cnt.p, 0, sizeof(int) * ncnt, ctx->stream));
	W.nwork = (int)list.size();
	W.work = dlist;
	W.next = ctx->wl_cnt.p;
	W.cnt = ctx->wl_cnt.p + 1;
	W.errflag = ctx->errflag.p;
	int npq32 = 1;
	for (int i = 0; i < W.nseg; i++)
		if (W.seg[i].n == 32) npq32 = std::max(npq32, W.seg[i].npq);
	using WlKernel = void (*)(const WorkParams);
	const WlKernel kern = half32
		? (npq32 == 1 ? (WlKernel)worklist_kernel<1, true> : npq32 == 2 ? (WlKernel)worklist_kernel<2, true> : (WlKernel)worklist_kernel<4, true>)
		: (npq32 == 1 ? (WlKernel)worklist_kernel<1, false> : npq32 == 2 ? (WlKernel)worklist_kernel<2, false> : (WlKernel)worklist_kernel<4, false>);
	const int kv = (npq32 == 1 ? 0 : npq32 == 2 ? 1 : 2) + (half32 ? 3 : 0);
	static int resident[64][6] = {{0}};
	if (ctx->device >= 64) return fail(ctx, SHWFS_EINVAL, "work list: device %d out of range", ctx->device);
	if (!resident[ctx->device][kv]) {
		CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, WL_N32_SMEM));
		int per_sm = 0, nsm = 0;
		CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WL_THREADS, WL_N32_SMEM));
		CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
		resident[ctx->device][kv] = std::max(1, per_sm) * nsm;
	}
	// no more blocks than the device holds at once: a wait only ever depends on
	// items already handed to running blocks
	const int grid = std::min(W.nwork, resident[ctx->device][kv]);
	{
		StageMark mark(ctx, SHWFS_STAGE_INTS);
		kern<<<grid, WL_THREADS, WL_N32_SMEM, ctx->stream>>>(W);
		ctx->errflag_armed = 1;
	}
	CK(cudaGetLastError());
	return 0;
}

int shwfs_set_worklist(shwfs_ctx* ctx, int on, int slices, int group) {
	if (!ctx || slices < 0 || group < 0 || group > 64)
		return ctx ? fail(ctx, SHWFS_EINVAL, "set_worklist: bad arguments") : SHWFS_EINVAL;
	ctx->worklist = on ? 1 : 0;
	if (slices) ctx->wl_slices = slices;
	if (group) ctx->wl_group = group;
	ctx->g_warm = 0;  // a frame graph is captured again
	return 0;
}

// Destroys the powfs branches and the frame graph (made again by the next frame).
static int drop_branches(shwfs_ctx* ctx) {
	// the branches are made again, at the new priorities, by the next frame
	for (size_t i = 0; i < ctx->pstream.size(); i++) {
		CK(cudaStreamSynchronize(ctx->pstream[i]));
		CK(cudaStreamDestroy(ctx->pstream[i]));
		CK(cudaEventDestroy(ctx->ev_pfork[i]));
		CK(cudaEventDestroy(ctx->ev_pjoin[i]));
	}
	ctx->pstream.clear();
	ctx->ev_pfork.clear();
	ctx->ev_pjoin.clear();
	if (ctx->gexec) {
		CK(cudaGraphExecDestroy(ctx->gexec));
		ctx->gexec = nullptr;
	}
	ctx->g_warm = 0;
	return 0;
}

int shwfs_set_branch_priority(shwfs_ctx* ctx, int on) {
	if (!ctx) return SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	CK(cudaStreamSynchronize(ctx->stream));
	if ((r = drop_branches(ctx))) return r;
	ctx->branch_priority = on ? 1 : 0;
	return 0;
}

int shwfs_set_stream_priority(shwfs_ctx* ctx, int priority) {
	if (!ctx) return SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	int lo = 0, hi = 0;
	CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
	const int p = std::min(lo, std::max(hi, priority));
	CK(cudaStreamSynchronize(ctx->stream));
	CK(cudaStreamSynchronize(ctx->aux));
	if ((r = drop_branches(ctx))) return r;
	cudaStream_t s = nullptr, a = nullptr;
	CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, p));
	if (cudaStreamCreateWithPriority(&a, cudaStreamNonBlocking, hi) != cudaSuccess) {
		cudaStreamDestroy(s);
		return fail(ctx, SHWFS_ECUDA, "set_stream_priority: stream creation failed");
	}
	CK(cudaStreamDestroy(ctx->stream));
	CK(cudaStreamDestroy(ctx->aux));
	ctx->stream = s;
	ctx->aux = a;
	ctx->priority = p;
	return 0;
}

int shwfs_frame_queue(shwfs_ctx* ctx, int isim, int iwfs0, int iwfs1) {
	if (!ctx || iwfs0 < 0 || iwfs1 > (int)ctx->wfs.size() || iwfs0 >= iwfs1)
		return ctx ? fail(ctx, SHWFS_EINVAL, "frame_queue: bad WFS range") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	std::vector<std::vector<int>> wl(ctx->powfs.size());
	int nbranch = 0;
	for (size_t ip = 0; ip < ctx->powfs.size(); ip++) {
		for (int i = iwfs0; i < iwfs1; i++)
			if (ctx->wfs[i].d.ipowfs == (int)ip) {
				if ((r = check_ready(ctx, ctx->powfs[ip], ctx->wfs[i]))) return r;
				wl[ip].push_back(i);
			}
		if (!wl[ip].empty()) nbranch++;
	}
	ctx->cache_desc = 1;
	if (ctx->worklist) {
		r = frame_worklist(ctx, wl, isim);
		if (r <= 0) {
			ctx->cache_desc = 0;
			return r;
		}
		r = 0;  // a powfs the work list does not serve: the ordinary frame
	}
	if (nbranch <= 1) {
		for (size_t ip = 0; ip < ctx->powfs.size() && !r; ip++)
			if (!wl[ip].empty()) r = frame_powfs(ctx, (int)ip, wl[ip], isim);
		ctx->cache_desc = 0;
		return r;
	}
	// several powfs: each on its own branch, so the small sensors' chains run
	// beside the large ones
	if (!ctx->capturing && (r = ensure_branches(ctx))) {
		ctx->cache_desc = 0;
		return r;
	}
	if (ctx->pstream.size() < ctx->powfs.size()) {
		ctx->cache_desc = 0;
		return fail(ctx, SHWFS_ESTATE, "frame graph: stream branches not created by a warm-up frame");
	}
	cudaStream_t main = ctx->stream;
	CK(cudaEventRecord(ctx->ev_pfork[0], main));
	for (size_t ip = 0; ip < ctx->powfs.size(); ip++) {
		if (wl[ip].empty()) continue;
		CK(cudaStreamWaitEvent(ctx->pstream[ip], ctx->ev_pfork[0], 0));
		ctx->stream = ctx->pstream[ip];
		if (!r) r = frame_powfs(ctx, (int)ip, wl[ip], isim);
		ctx->stream = main;
		CK(cudaEventRecord(ctx->ev_pjoin[ip], ctx->pstream[ip]));
		CK(cudaStreamWaitEvent(main, ctx->ev_pjoin[ip], 0));
	}
	ctx->cache_desc = 0;
	return r;
}

int shwfs_frame_graph(shwfs_ctx* ctx, int isim, int iwfs0, int iwfs1) {
	if (!ctx || iwfs0 < 0 || iwfs1 > (int)ctx->wfs.size() || iwfs0 >= iwfs1)
		return ctx ? fail(ctx, SHWFS_EINVAL, "frame_graph: bad WFS range") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (ctx->profiling) return fail(ctx, SHWFS_ESTATE, "frame_graph: stage profiling must be off");
	if (!ctx->g_warm || ctx->g_i0 != iwfs0 || ctx->g_i1 != iwfs1) {
		// warm-up frame: buffers, descriptor cache and stream branches come into being
		if ((r = shwfs_frame_queue(ctx, isim, iwfs0, iwfs1))) return r;
		if (ctx->gexec) {
			CK(cudaGraphExecDestroy(ctx->gexec));
			ctx->gexec = nullptr;
		}
		ctx->g_warm = 1;
		ctx->g_i0 = iwfs0;
		ctx->g_i1 = iwfs1;
		return 0;
	}
	cudaGraph_t g = nullptr;
	CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
	ctx->capturing = 1;
	r = shwfs_frame_queue(ctx, isim, iwfs0, iwfs1);
	ctx->capturing = 0;
	const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
	if (r || e != cudaSuccess) {
		if (g) cudaGraphDestroy(g);
		ctx->g_warm = 0;
		return r ? r : fail(ctx, SHWFS_ECUDA, "frame_graph: capture failed: %s", cudaGetErrorString(e));
	}
	if (ctx->gexec) {
		cudaGraphExecUpdateResultInfo info;
		if (cudaGraphExecUpdate(ctx->gexec, g, &info) != cudaSuccess) {
			cudaGetLastError();
			CK(cudaGraphExecDestroy(ctx->gexec));
			ctx->gexec = nullptr;
		}
	}
	if (!ctx->gexec) {
		// the branches' stream priorities, captured as node priorities, hold in the graph
		const cudaError_t ei = cudaGraphInstantiate(&ctx->gexec, g, cudaGraphInstantiateFlagUseNodePriority);
		if (ei != cudaSuccess) {
			cudaGraphDestroy(g);
			ctx->gexec = nullptr;
			return fail(ctx, SHWFS_ECUDA, "frame_graph: instantiate: %s", cudaGetErrorString(ei));
		}
	}
	CK(cudaGraphDestroy(g));
	CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
	return 0;
}

int shwfs_frame_sync(shwfs_ctx* ctx, int iwfs, double* grad, double* ints) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "frame_sync: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	const int nsa = p.d.nsa, npix = p.d.pixpsax * p.d.pixpsay;
	if (ints && is_geom(p.d.gradtype)) return fail(ctx, SHWFS_EINVAL, "frame_sync: geometric sensor has no pixels");
	if (grad) {
		CK(cudaMemcpyAsync(w->grad_h, w->grad.p, sizeof(float) * 2 * nsa, cudaMemcpyDeviceToHost, ctx->stream));
		ctx->d2h_bytes += sizeof(float) * 2 * nsa;
	}
	if (ints) {
		CK(cudaMemcpyAsync(w->ints_h, w->ints.p, sizeof(float) * nsa * npix, cudaMemcpyDeviceToHost, ctx->stream));
		ctx->d2h_bytes += sizeof(float) * nsa * npix;
	}
	// the error flag travels only when a kernel that can set it ran since the last check
	const bool chk = ctx->errflag.p && ctx->errflag_armed;
	if (chk) {
		if (!ctx->errflag_h) CK(cudaMallocHost(&ctx->errflag_h, sizeof(int)));
		CK(cudaMemcpyAsync(ctx->errflag_h, ctx->errflag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
	}
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->wfsdev_h.clear();
	if (chk) {
		ctx->errflag_armed = 0;
		if (*ctx->errflag_h) {
			CK(cudaMemset(ctx->errflag.p, 0, sizeof(int)));
			return fail(ctx, SHWFS_ETIMEOUT, "a bounded device wait expired in an imaging kernel");
		}
	}
	if (grad) f32_to_f64(w->grad_h, grad, (size_t)2 * nsa);
	if (ints) f32_to_f64(w->ints_h, ints, (size_t)nsa * npix);
	return 0;
}

int shwfs_wfs_update_mtche(shwfs_ctx* ctx, int iwfs, int mtchcr) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || mtchcr < 0 || mtchcr > 3) return ctx ? fail(ctx, SHWFS_EINVAL, "update_mtche: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	const shwfs_powfs_desc& d = p.d;
	const int nsa = d.nsa, npix = d.pixpsax * d.pixpsay;
	if (!(d.nopd == 16 && d.notf == 32)) return fail(ctx, SHWFS_EINVAL, "update_mtche: needs 16x16 OPD points and FFT 32");
	if (d.gradtype != SHWFS_GRAD_MF) return fail(ctx, SHWFS_EINVAL, "update_mtche: the powfs uses CoG gradients");
	if (!p.bands.empty()) return fail(ctx, SHWFS_EINVAL, "update_mtche: a powfs of several wavelength bands takes its filter from the host");
	if (p.nsimap != 1 || npix > 128) return fail(ctx, SHWFS_EINVAL, "update_mtche: needs one pixel map of at most 128 pixels");
	if (!p.amp.p || !p.simap_idx.p) return fail(ctx, SHWFS_ESTATE, "update_mtche: geometry or pixel map not set");
	if (d.has_etf ? !p.etfT[0].p : !p.nominalT.p) return fail(ctx, SHWFS_ESTATE, "update_mtche: ETF / DTF not set");
	if (!p.zero_opd.p) {
		std::vector<float> z(256, 0.f);
		if ((r = dev_upload(ctx, p.zero_opd, z.data(), z.size()))) return r;
	}
	const bool se = p.seotfT.p != nullptr;  // the short-exposure OTF of shwfs_powfs_set_seotf
	if (!se && d.has_llt && !p.lotf_flat.p) {  // without it: the flat uplink OTF
		if (!p.lltamp.p) return fail(ctx, SHWFS_ESTATE, "update_mtche: LLT amplitude not set");
		if ((r = dev_alloc(ctx, p.lotf_flat, (size_t)d.notf * d.notf))) return r;
		DevBuf<const float*> in;
		DevBuf<float2*> out;
		const float* zi = p.zero_opd.p;
		float2* zo = p.lotf_flat.p;
		if ((r = dev_upload(ctx, in, &zi, 1)) || (r = dev_upload(ctx, out, &zo, 1))) return r;
		uplink_otf_n32_kernel<<<1, 128, 0, ctx->stream>>>(in.p, p.lltamp.p, out.p, 1, 0.f,
			(float)(1.0 / ((double)d.llt_nx * d.embfac * d.llt_nx * d.embfac)));
		CK(cudaGetLastError());
		CK(cudaStreamSynchronize(ctx->stream));
		in.free_();
		out.free_();
	}
	if ((r = dev_alloc(ctx, p.mtch_img, (size_t)nsa * 3 * npix)) || (r = dev_alloc(ctx, p.mtch_red, 2))) return r;
	if (!w->mtche.p && (r = dev_alloc(ctx, w->mtche, (size_t)nsa * 2 * npix))) return r;
	if (!w->i0sum.p && (r = dev_alloc(ctx, w->i0sum, (size_t)nsa))) return r;
	CK(cudaMemsetAsync(p.mtch_red.p, 0, 2 * sizeof(double), ctx->stream));
	const PowfsDev P = make_powfs_dev(p, 0);
	MtchParams M;
	memset(&M, 0, sizeof(M));
	M.nsa = nsa;
	M.npix = npix;
	M.pixpsax = d.pixpsax;
	M.pixpsay = d.pixpsay;
	M.nmod = 3;
	if (mtchcr == 1 || mtchcr == 2) {
		M.crx = M.nmod;
		M.nmod += 2;
	}
	if (mtchcr == 1 || mtchcr == 3) {
		M.cry = M.nmod;
		M.nmod += 2;
	}
	// gensei (lib/gensei.c:320-366) scales the short-exposure images by the signal level alone
	M.norm_ints = se ? (float)(w->d.sigsim * w->d.wvlwt) : norm_ints(p, *w);
	M.seotfT = se ? p.seotfT.p : nullptr;
	M.dux = (float)(1.0 / (d.wvl / (d.dsa * d.embfac) * d.notf));
	M.amp = p.amp.p + (p.namp > 1 ? (size_t)w->wfsind * nsa * 256 : 0);
	M.zero_opd = p.zero_opd.p;
	M.lotfT = d.has_llt ? p.lotf_flat.p : nullptr;
	M.etfT1 = P.etfT1;
	M.etfT2 = P.etfT2;
	M.etfwt1 = P.etfwt1;
	M.etfwt2 = P.etfwt2;
	M.nominalT = P.nominalT;
	M.nominal_per_sa = P.nominal_per_sa;
	M.simap_idx = p.simap_idx.p;
	M.simap_wt = p.simap_wt.p;
	M.kpx = 1. / d.pixthetax;
	M.kpy = 1. / d.pixthetay;
	M.bkgrnd = d.bkgrnd;
	M.bkgrnd_res = d.bkgrnd - d.bkgrndc;
	M.rne = d.rne;
	M.nea2thres = d.pixthetax * d.pixthetax * 100;
	M.img = p.mtch_img.p;
	M.i0sum = w->i0sum.p;
	M.i0sumsum = p.mtch_red.p;
	M.i0max_bits = reinterpret_cast<unsigned*>(p.mtch_red.p + 1);
	M.mtche = w->mtche.p;
	const int nblk = (nsa + 3) / 4;
	if (npix <= 32) {
		mtch_images_kernel<1><<<nblk, 128, 0, ctx->stream>>>(M);
		mtch_filter_kernel<1><<<nblk, 128, 0, ctx->stream>>>(M);
	} else if (npix <= 64) {
		mtch_images_kernel<2><<<nblk, 128, 0, ctx->stream>>>(M);
		mtch_filter_kernel<2><<<nblk, 128, 0, ctx->stream>>>(M);
	} else {
		mtch_images_kernel<4><<<nblk, 128, 0, ctx->stream>>>(M);
		mtch_filter_kernel<4><<<nblk, 128, 0, ctx->stream>>>(M);
	}
	CK(cudaGetLastError());
	double tot = 0;
	CK(cudaMemcpyAsync(&tot, p.mtch_red.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	w->i0sumsum = tot;
	return check_errflag(ctx);
}

int shwfs_powfs_set_etf_dtrat(shwfs_ctx* ctx, int ipowfs, int dtrat) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || dtrat < 0) return ctx ? fail(ctx, SHWFS_EINVAL, "set_etf_dtrat: bad arguments") : SHWFS_EINVAL;
	if (dtrat > 0 && !p->d.has_etf) return fail(ctx, SHWFS_EINVAL, "set_etf_dtrat: the powfs has no ETF");
	p->etf_dtrat = dtrat;
	return 0;
}

int shwfs_powfs_set_dtrat(shwfs_ctx* ctx, int ipowfs, int dtrat) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || dtrat < 1 || dtrat > 100000) return ctx ? fail(ctx, SHWFS_EINVAL, "set_dtrat: bad arguments") : SHWFS_EINVAL;
	if (is_geom(p->d.gradtype) && dtrat > 1) return fail(ctx, SHWFS_EINVAL, "set_dtrat: geometric sensors form every frame");
	if (p->d.sigmatch == 2 && dtrat > 1) return fail(ctx, SHWFS_EINVAL, "set_dtrat: sigmatch 2 with dtrat > 1 is not supported");
	if (p->band_of >= 0) return fail(ctx, SHWFS_EINVAL, "set_dtrat: a wavelength band integrates with its powfs %d", p->band_of);
	p->dtrat = dtrat;
	return 0;
}

int shwfs_powfs_set_saasum(shwfs_ctx* ctx, int ipowfs, double saasum) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || !(saasum > 0)) return ctx ? fail(ctx, SHWFS_EINVAL, "set_saasum: bad arguments") : SHWFS_EINVAL;
	p->saasum = saasum;
	return 0;
}

int shwfs_wfs_set_neasim(shwfs_ctx* ctx, int iwfs, const double* nea) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w) return ctx ? fail(ctx, SHWFS_EINVAL, "set_neasim: unknown wfs %d", iwfs) : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (!nea) {
		w->neasim.free_();
		return 0;
	}
	return dev_upload_f(ctx, w->neasim, nea, (size_t)3 * ctx->powfs[w->d.ipowfs].d.nsa);
}

int shwfs_grad_ztilt_dev(shwfs_ctx* ctx, int iwfs, const float* opd, float* grad) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || !opd || !grad) return ctx ? fail(ctx, SHWFS_EINVAL, "grad_ztilt: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const PowfsState& p = ctx->powfs[w->d.ipowfs];
	if (!p.amp.p || !p.origx.p) return fail(ctx, SHWFS_ESTATE, "powfs geometry not set");
	// the z-tilt fit on any powfs's geometry
	const int nsa = p.d.nsa;
	const float* amp = p.amp.p + (p.namp > 1 ? (size_t)w->wfsind * nsa * p.d.nopd * p.d.nopd : 0);
	ztilt_kernel<<<(nsa + 7) / 8, 256, 0, ctx->stream>>>(opd, amp, p.origx.p, p.origy.p, nsa, p.d.nopd, p.d.dx, grad,
		nullptr, 0, 0, 0);
	CK(cudaGetLastError());
	return 0;
}

int shwfs_grad_gtilt_dev(shwfs_ctx* ctx, int iwfs, const float* opd, float* grad) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || !opd || !grad) return ctx ? fail(ctx, SHWFS_EINVAL, "grad_gtilt: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	if (ctx->powfs[w->d.ipowfs].d.gradtype != SHWFS_GRAD_GTILT)
		return fail(ctx, SHWFS_EINVAL, "grad_gtilt: the powfs is not a G-tilt sensor");
	return launch_geom_grad(ctx, *w, opd, grad, false, 0);
}

int shwfs_powfs_set_gs0(shwfs_ctx* ctx, int ipowfs, int iamp, long nrow, long ncol, const int* pp, const int* pi,
	const double* px) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || iamp < 0 || iamp > 1023 || !pp || (pp[ncol] > 0 && (!pi || !px)))
		return ctx ? fail(ctx, SHWFS_EINVAL, "set_gs0: bad arguments") : SHWFS_EINVAL;
	const long nsa = p->d.nsa, nloc = (long)nsa * p->d.nopd * p->d.nopd;
	if (nrow != 2 * nsa || ncol != nloc)
		return fail(ctx, SHWFS_EINVAL, "set_gs0: GS0 is %ldx%ld, needs %ldx%ld", nrow, ncol, 2 * nsa, nloc);
	// CSC (MAOS dsp) -> CSR, checking every index
	const long nnz = pp[ncol];
	if (pp[0] != 0 || nnz < 0 || nnz > 0x7fffffffL) return fail(ctx, SHWFS_EINVAL, "set_gs0: bad column pointers");
	std::vector<int> rp(nrow + 1, 0), ci(nnz);
	std::vector<double> v(nnz);
	for (long c = 0; c < ncol; c++) {
		if (pp[c + 1] < pp[c] || pp[c + 1] > nnz) return fail(ctx, SHWFS_EINVAL, "set_gs0: bad column pointers");
		for (long k = pp[c]; k < pp[c + 1]; k++) {
			if (pi[k] < 0 || pi[k] >= nrow) return fail(ctx, SHWFS_EINVAL, "set_gs0: row index out of range");
			rp[pi[k] + 1]++;
		}
	}
	for (long i = 0; i < nrow; i++) rp[i + 1] += rp[i];
	std::vector<int> fill(rp.begin(), rp.end() - 1);
	for (long c = 0; c < ncol; c++)
		for (long k = pp[c]; k < pp[c + 1]; k++) {
			const int at = fill[pi[k]]++;
			ci[at] = (int)c;
			v[at] = px[k];
		}
	int r = set_device(ctx);
	if (r) return r;
	if ((size_t)iamp >= p->gs0_ptr.size()) {
		p->gs0_ptr.resize(iamp + 1);
		p->gs0_col.resize(iamp + 1);
		p->gs0_val.resize(iamp + 1);
	}
	if ((r = dev_upload(ctx, p->gs0_ptr[iamp], rp.data(), rp.size()))) return r;
	if (nnz == 0) return 0;
	if ((r = dev_upload(ctx, p->gs0_col[iamp], ci.data(), ci.size()))) return r;
	return dev_upload_f(ctx, p->gs0_val[iamp], v.data(), v.size());
}

int shwfs_frame_sync_range(shwfs_ctx* ctx, int iwfs0, int iwfs1, double* grad) {
	if (!ctx || !grad || iwfs0 < 0 || iwfs1 > (int)ctx->wfs.size() || iwfs0 >= iwfs1)
		return ctx ? fail(ctx, SHWFS_EINVAL, "frame_sync_range: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	// one copy per run of WFS whose gradients are consecutive in an arena chunk
	for (int i = iwfs0; i < iwfs1;) {
		const WfsState& w0 = ctx->wfs[i];
		size_t n = w0.grad.n;
		int j = i + 1;
		while (j < iwfs1 && w0.garena >= 0 && ctx->wfs[j].garena == w0.garena && ctx->wfs[j].grad.p == w0.grad.p + n) {
			n += ctx->wfs[j].grad.n;
			j++;
		}
		CK(cudaMemcpyAsync(w0.grad_h, w0.grad.p, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
		ctx->d2h_bytes += sizeof(float) * n;
		i = j;
	}
	// the error flag travels only when a kernel that can set it ran since the last check
	const bool chk = ctx->errflag.p && ctx->errflag_armed;
	if (chk) {
		if (!ctx->errflag_h) CK(cudaMallocHost(&ctx->errflag_h, sizeof(int)));
		CK(cudaMemcpyAsync(ctx->errflag_h, ctx->errflag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
	}
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->wfsdev_h.clear();
	if (chk) {
		ctx->errflag_armed = 0;
		if (*ctx->errflag_h) {
			CK(cudaMemset(ctx->errflag.p, 0, sizeof(int)));
			return fail(ctx, SHWFS_ETIMEOUT, "a bounded device wait expired in an imaging kernel");
		}
	}
	for (int i = iwfs0; i < iwfs1; i++) {
		const size_t n = ctx->wfs[i].grad.n;
		f32_to_f64(ctx->wfs[i].grad_h, grad, n);
		grad += n;
	}
	return 0;
}

int shwfs_autotune(shwfs_ctx* ctx, int iwfs0, int iwfs1, int nrep, int* chosen) {
	if (!ctx || iwfs0 < 0 || iwfs1 > (int)ctx->wfs.size() || iwfs0 >= iwfs1 || nrep <= 0)
		return ctx ? fail(ctx, SHWFS_EINVAL, "autotune: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	const int ipowfs = ctx->wfs[iwfs0].d.ipowfs;
	PowfsState& p = ctx->powfs[ipowfs];
	// whole frames on the device: the variants differ in which launches a frame has
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	CK(cudaEventCreate(&e0));
	if (cudaEventCreate(&e1) != cudaSuccess) {
		cudaEventDestroy(e0);
		return fail(ctx, SHWFS_ECUDA, "autotune: cudaEventCreate failed");
	}
	double best = 1e300;
	int bestv = 0;
	for (int v = 0; v < SHWFS_NVARIANT && !r; v++) {
		p.variant = v;
		if ((r = shwfs_frame_queue(ctx, 0, iwfs0, iwfs1))) break;  // warm
		if (cudaEventRecord(e0, ctx->stream) != cudaSuccess) { r = fail(ctx, SHWFS_ECUDA, "autotune: event record failed"); break; }
		for (int k = 0; k < nrep && !r; k++) r = shwfs_frame_queue(ctx, k, iwfs0, iwfs1);
		if (r) break;
		float ms = 0.f;
		if (cudaEventRecord(e1, ctx->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
			cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
			r = fail(ctx, SHWFS_ECUDA, "autotune: event timing failed");
			break;
		}
		if (ms < best) {
			best = ms;
			bestv = v;
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (r) return r;
	p.variant = bestv;
	if (chosen) *chosen = bestv;
	return 0;
}

// The frame layouts shwfs_autotune_frame compares: per-powfs launches, then the
// work list at these (slices, group).
static const int kWlChoices[][2] = {{7, 4}, {14, 4}, {28, 4}, {7, 8}};
constexpr int WL_NCHOICE = 1 + (int)(sizeof(kWlChoices) / sizeof(kWlChoices[0]));

int shwfs_autotune_frame(shwfs_ctx* ctx, int iwfs0, int iwfs1, int nrep, int* choice) {
	if (!ctx || iwfs0 < 0 || iwfs1 > (int)ctx->wfs.size() || iwfs0 >= iwfs1 || nrep <= 0)
		return ctx ? fail(ctx, SHWFS_EINVAL, "autotune_frame: bad arguments") : SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	CK(cudaEventCreate(&e0));
	if (cudaEventCreate(&e1) != cudaSuccess) {
		cudaEventDestroy(e0);
		return fail(ctx, SHWFS_ECUDA, "autotune_frame: cudaEventCreate failed");
	}
	double best = 1e300;
	int bestc = 0;
	// frames as CUDA graphs, the form in which a frame of several powfs runs
	// free of host launch costs (a layout of many small launches would lose to
	// one of few launches only through the host); stream frames while stage
	// profiling is on, which graphs do not allow
	auto frame = [&](int k) {
		return ctx->profiling ? shwfs_frame_queue(ctx, k, iwfs0, iwfs1) : shwfs_frame_graph(ctx, k, iwfs0, iwfs1);
	};
	for (int c = 0; c < WL_NCHOICE && !r; c++) {
		ctx->worklist = c > 0;
		if (c > 0) {
			ctx->wl_slices = kWlChoices[c - 1][0];
			ctx->wl_group = kWlChoices[c - 1][1];
		}
		ctx->g_warm = 0;  // the layout's own graph: a warm-up frame, then a capture
		if ((r = frame(0)) || (r = frame(1))) break;
		if (cudaEventRecord(e0, ctx->stream) != cudaSuccess) { r = fail(ctx, SHWFS_ECUDA, "autotune_frame: event record failed"); break; }
		for (int k = 0; k < nrep && !r; k++) r = frame(2 + k);
		if (r) break;
		float ms = 0.f;
		if (cudaEventRecord(e1, ctx->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
			cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
			r = fail(ctx, SHWFS_ECUDA, "autotune_frame: event timing failed");
			break;
		}
		if (ms < best) {
			best = ms;
			bestc = c;
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (r) return r;
	ctx->worklist = bestc > 0;
	if (bestc > 0) {
		ctx->wl_slices = kWlChoices[bestc - 1][0];
		ctx->wl_group = kWlChoices[bestc - 1][1];
	}
	ctx->g_warm = 0;
	if (choice) *choice = bestc;
	return 0;
}

int shwfs_set_trace_order(shwfs_ctx* ctx, int order) {
	if (!ctx) return SHWFS_EINVAL;
	if (order < SHWFS_TRACE_AUTO || order > SHWFS_TRACE_INTERLEAVED)
		return fail(ctx, SHWFS_EINVAL, "set_trace_order: order %d is not AUTO, LISTED or INTERLEAVED", order);
	ctx->trace_order = order;
	return 0;
}

int shwfs_set_variant(shwfs_ctx* ctx, int ipowfs, int variant) {
	PowfsState* p = get_powfs(ctx, ipowfs);
	if (!p || variant < 0 || variant >= SHWFS_NVARIANT) return ctx ? fail(ctx, SHWFS_EINVAL, "set_variant: bad arguments") : SHWFS_EINVAL;
	p->variant = variant;
	return 0;
}

int shwfs_copy_counters(shwfs_ctx* ctx, uint64_t* h2d, uint64_t* d2h) {
	if (!ctx) return SHWFS_EINVAL;
	if (h2d) *h2d = ctx->h2d_bytes;
	if (d2h) *d2h = ctx->d2h_bytes;
	ctx->h2d_bytes = ctx->d2h_bytes = 0;
	return 0;
}

int shwfs_profile_enable(shwfs_ctx* ctx, int enable) {
	if (!ctx) return SHWFS_EINVAL;
	ctx->profiling = enable ? 1 : 0;
	return 0;
}

int shwfs_profile_read(shwfs_ctx* ctx, double* ms, int* launches) {
	if (!ctx || !ms || !launches) return SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	CK(cudaStreamSynchronize(ctx->stream));
	CK(cudaStreamSynchronize(ctx->aux));
	for (int i = 0; i < SHWFS_NSTAGE; i++) {
		ms[i] = 0;
		launches[i] = 0;
	}
	for (auto& m : ctx->marks) {
		float t = 0;
		CK(cudaEventElapsedTime(&t, m.a, m.b));
		ms[m.stage] += t;
		launches[m.stage]++;
		ctx->ev_pool.push_back(m.a);
		ctx->ev_pool.push_back(m.b);
	}
	ctx->marks.clear();
	return 0;
}

int shwfs_sync(shwfs_ctx* ctx) {
	if (!ctx) return SHWFS_EINVAL;
	int r = set_device(ctx);
	if (r) return r;
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->wfsdev_h.clear();
	return check_errflag(ctx);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free frame.
//
// For callers that must not allocate device memory once they run: a
// real-time control loop that forbids allocation after start-up (an
// allocation can block for milliseconds and fail when memory is short), or a
// host application whose device memory is handed out by its own pool.  The
// ordinary frame keeps its scratch (the ray-traced OPD,
// the LLT OPD, the uplink OTF and the launch descriptor) in buffers the
// context allocates; this variant keeps them in one file-scope device array
// instead, so a call allocates nothing.
//
// The array is SHWFS_NOALLOC_SCRATCH_FLOATS floats (about 4 MiB) and every
// GPU that loads the library holds it until the process exits.  Its host-side
// name is only a stand-in for the device symbol, so the device address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current, the first time the entry point runs on it.  All calls on a device
// share the array: every element a call reads is first written by the same
// call, so nothing needs clearing between calls, but calls whose work
// overlaps on the GPU (two streams, two contexts, two threads) race on it.
// ---------------------------------------------------------------------------
#include <mutex>

#define NOALLOC_OPD_FLOATS (SHWFS_NOALLOC_MAX_NSA * 256)
#define NOALLOC_LLT_OFF NOALLOC_OPD_FLOATS
#define NOALLOC_LOTF_OFF (NOALLOC_LLT_OFF + 256)
#define NOALLOC_DESC_OFF (NOALLOC_LOTF_OFF + 2048)
#define SHWFS_NOALLOC_SCRATCH_FLOATS (NOALLOC_DESC_OFF + 64)

static __device__ __align__(256) float g_noalloc_scratch[SHWFS_NOALLOC_SCRATCH_FLOATS];

namespace {
std::mutex g_noalloc_mutex;
float* g_noalloc_ptr[64] = {nullptr};
}  // namespace

__global__ void noalloc_desc_kernel(WfsDev wd, WfsDev* dst) { *dst = wd; }

static int noalloc_scratch(shwfs_ctx* ctx, float** out) {
	if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, SHWFS_EINVAL, "frame_noalloc: device %d out of range", ctx->device);
	std::lock_guard<std::mutex> lock(g_noalloc_mutex);
	if (!g_noalloc_ptr[ctx->device]) {
		void* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p)
			return fail(ctx, SHWFS_ECUDA, "frame_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
		g_noalloc_ptr[ctx->device] = (float*)p;
	}
	*out = g_noalloc_ptr[ctx->device];
	return 0;
}

extern "C" {

int shwfs_frame_noalloc(shwfs_ctx* ctx, int iwfs, int isim, float* ints, float* grad) {
	WfsState* w = get_wfs(ctx, iwfs);
	if (!w || (!ints && !grad)) return ctx ? fail(ctx, SHWFS_EINVAL, "frame_noalloc: bad arguments") : SHWFS_EINVAL;
	PowfsState& p = ctx->powfs[w->d.ipowfs];
	if (is_geom(p.d.gradtype)) return fail(ctx, SHWFS_EINVAL, "frame_noalloc: geometric sensor");
	if (p.d.sigmatch == 2) return fail(ctx, SHWFS_EINVAL, "frame_noalloc: sigmatch 2 needs the frame path");
	if (p.dtrat > 1) return fail(ctx, SHWFS_EINVAL, "frame_noalloc: dtrat > 1 needs the frame path");
	if (!p.bands.empty()) return fail(ctx, SHWFS_EINVAL, "frame_noalloc: wavelength bands need the frame path");
	if (p.d.nsa > SHWFS_NOALLOC_MAX_NSA)
		return fail(ctx, SHWFS_EINVAL, "frame_noalloc: %d subapertures exceed the allocation-free maximum of %d",
			p.d.nsa, SHWFS_NOALLOC_MAX_NSA);
	// the scratch offsets, the 32x32 image tile of ints_n32_kernel and the fused
	// uplink all assume the 32-point form: 16x16 OPD points padded to a 32x32 FFT
	if (!(p.d.nopd == 16 && p.d.nopd * p.d.embfac == 32 && p.d.notf == 32))
		return fail(ctx, SHWFS_EINVAL,
			"frame_noalloc: only 16x16 OPD points with a 32x32 FFT are served (this powfs: n_opd=%d n_w=%d n_f=%d)",
			p.d.nopd, p.d.nopd * p.d.embfac, p.d.notf);
	if (p.d.pixpsax * p.d.pixpsay > 128)
		return fail(ctx, SHWFS_EINVAL, "frame_noalloc: at most 128 pixels per subaperture");
	int r = set_device(ctx);
	if (r) return r;
	if ((r = check_ready(ctx, p, *w))) return r;
	float* scratch = nullptr;
	if ((r = noalloc_scratch(ctx, &scratch))) return r;
	// stage timing would create CUDA events: keep it off for this call
	struct ProfileOff {
		shwfs_ctx* c;
		int saved;
		~ProfileOff() { c->profiling = saved; }
	} prof_off{ctx, ctx->profiling};
	ctx->profiling = 0;
	float* opd = scratch;
	float* lltopd = scratch + NOALLOC_LLT_OFF;
	float2* lotfT = reinterpret_cast<float2*>(scratch + NOALLOC_LOTF_OFF);
	WfsDev* desc = reinterpret_cast<WfsDev*>(scratch + NOALLOC_DESC_OFF);
	// (a) ray trace (and the LGS uplink) into the scratch array
	GeomParams gp;
	geom_init(ctx, gp);
	if ((r = add_wfs_entry(ctx, gp, *w, isim, opd))) return r;
	if (p.d.has_llt) {
		if ((r = add_geom_entry(ctx, gp, w->d.thetax - p.d.llt_ox / w->d.hs, w->d.thetay - p.d.llt_oy / w->d.hs, w->d.hs,
				 0, 0, 0, p.d.llt_ox, p.d.llt_oy, isim, p.lltorig.p, p.lltorig.p + 1, 1, p.d.llt_nx, p.d.dx, lltopd)))
			return r;
		GeomEntry& e = gp.e[gp.nentry - 1];
		set_llt_poly(e, *w);
		e.lltamp = p.lltamp.p;
		e.lotfT = lotfT;
		e.twoinvwvl = (float)(2.0 / p.d.wvl);
		e.lltnorm = (float)(1.0 / ((double)p.d.llt_nx * p.d.embfac * p.d.llt_nx * p.d.embfac));
	}
	if ((r = launch_geom(ctx, gp))) return r;
	// (b)-(e) with the launch descriptor written on the device
	WfsDev wd;
	memset(&wd, 0, sizeof(wd));
	wd.opd = opd;
	wd.amp = p.amp.p + (p.namp > 1 ? (size_t)w->wfsind * p.d.nsa * p.d.nopd * p.d.nopd : 0);
	wd.lotfT = p.d.has_llt ? lotfT : nullptr;
	wd.mtche = w->mtche.p;
	wd.i0sum = w->i0sum.p;
	wd.ints = ints;
	wd.grad = grad;
	wd.alpha = norm_ints(p, *w);
	wd.noisy = w->d.noisy;
	wd.wfs_id = (uint32_t)iwfs;
	wd.seed = w->seed;
	noalloc_desc_kernel<<<1, 1, 0, ctx->stream>>>(wd, desc);
	CK(cudaGetLastError());
	PowfsDev P = make_powfs_dev(p, isim);
	const int nitem = p.d.nsa, nblk = (nitem + 3) / 4;
	if (P.npix <= 32)
		ints_n32_kernel<1, 5, true><<<nblk, 128, 0, ctx->stream>>>(P, desc, 1, nitem);
	else if (P.npix <= 64)
		ints_n32_kernel<2, 5, true><<<nblk, 128, 0, ctx->stream>>>(P, desc, 1, nitem);
	else
		ints_n32_kernel<4, 5, true><<<nblk, 128, 0, ctx->stream>>>(P, desc, 1, nitem);
	CK(cudaGetLastError());
	return 0;
}

}  // extern "C"

#include "shwfs_evl_host.cuh"
