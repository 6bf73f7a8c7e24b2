// Tensor-core (tcgen05) form of the imaging stages (b)-(e), n_opd=16, n_f=32.
//
// Every transform of the subaperture chain is a real GEMM on the 5th-gen
// tensor cores with BF16 operands split in three terms (a*b ~ ah*bh + ah*bl +
// al*bh, x = xh + xl, xl = bf16(x - xh)) and FP32 accumulators in TMEM:
//
//   2a  F1(x, ky)  = sum_y  E(x, y)  w32^(ky(y+8))     rows (s, x),  K = y   A in TMEM
//   2b  F(kx, ky)  = sum_x  F1(x,ky) w32^(kx(x+8))     rows (s, ky), K = x   A in smem, MN-major
//   4a  Q(ky, fx)  = sum_kx P(kx,ky) w32^(fx kx)       rows (s, ky), K = kx  A in TMEM  (P = |F|^2)
//   4b  O(fx, fy)  = sum_ky Q(ky,fx) w32^(fy ky)       rows (s, fx), K = ky  A in smem, MN-major
//   6a  T(fx, iy)  = sum_fy O'(fx,fy) Gy(iy, fy)       rows (s, fx), K = fy  A in TMEM  (O' = O x conj(uplink) x ETF)
//   6b  I(ix, iy)  = Re sum_fx T(fx,iy) Gx(ix, fx)     rows (s, iy), K = fx  A in smem, MN-major
//
// with w32 = exp(-2 pi i / 32) (FFTW's forward sign) and G = the inverse DFT
// premultiplied by the separable bilinear pixel weights, so the inverse
// transform and the pixel sampling of maos/wfsints.c:284-286 collapse into
// 6a/6b.  Complex operands are real blocks: K = [re | im], N = [re | im].
//
// Each stage leaves its output in TMEM, one GEMM row per lane.  Where that row
// is a row of the next A operand (field -> 2a, 2b -> 4a, 4b -> 6a) the lane
// writes it back to TMEM with tcgen05.st; where it is a K-row of the next A
// operand (2a -> 2b, 4a -> 4b, 6a -> 6b) the lane writes it to shared memory
// in the MN-major layout.  No stage transposes through shared memory.  The 6b
// rows (s, iy) with iy >= 8 read stale operand data and are never read back.
//
// A tile is 4 subapertures = 128 GEMM rows; warp w of a tile group owns
// subaperture w and TMEM lanes 32w..32w+31.  One CTA per SM holds four
// independent tile groups (4 warps each) that share the constant B operands,
// the WFS descriptors and the uplink OTFs in shared memory; each group has its
// own TMEM columns (64 accumulator + 64 A-operand), its own 32 KB MN-major
// operand buffer and its own mbarrier.  One thread per group issues the MMAs,
// commits them to the group's mbarrier and waits on it with a 2 s bound (on
// expiry the kernel records SHWFS_ETIMEOUT, frees its TMEM and returns); the
// rest of the group waits at a named barrier.  The kernel stores noise-free
// pixel intensities; photon/read noise and the gradients run in a separate
// one-warp-per-image kernel, whose occupancy hides their latency.
//
// Operand layouts (SWIZZLE_NONE, core matrices of 8 rows x 16 bytes):
//   K-major (B):  chunk (row r, k-chunk c) at ((r/8)*kc + c)*128 + (r%8)*16
//   MN-major (A): chunk (m-chunk mg, K-row k) at (mg*nkg + k/8)*128 + (k%8)*16
// LBO = 128 B is the stride along K, SBO the stride along M/N.  A TMEM A
// operand holds K pairs per 32-bit column (even K in the low half).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "shwfs_kernels.cuh"

namespace shwfs {

constexpr int SHWFS_ETIMEOUT_CODE = -5;  // SHWFS_ETIMEOUT of shwfs_b200.h

// ---- constants of the operand layouts ----
constexpr int TC_B1_BYTES = 64 * 8 * 16;   // N=64, K=32 (h|l: 8 chunks)   16-into-32 DFT
constexpr int TC_B2_BYTES = 64 * 16 * 16;  // N=64, K=64 (h|l: 16 chunks)  32-point DFT
constexpr int TC_B3_BYTES = 32 * 16 * 16;  // N=32 (16 re + 16 im pixel rows), K=64: Gy
constexpr int TC_B4_BYTES = 16 * 16 * 16;  // N=16 (pixel columns), K=64: [Re Gx | -Im Gx]
constexpr int TC_B_BYTES = TC_B1_BYTES + TC_B2_BYTES + TC_B3_BYTES + TC_B4_BYTES;
constexpr int TC_A_BYTES = 16 * 16 * 128;  // one group's MN-major A: 16 m-chunks x 16 k-groups
constexpr int TC_GROUPS = 4;               // tile groups per CTA (one CTA per SM)
constexpr int TC_THREADS = 128 * TC_GROUPS;
constexpr int TC_MAX_WFS = 6;              // WFS per launch (descriptors and uplink OTFs in smem)
constexpr int TC_LOTF_BYTES = 32 * 32 * 8; // one uplink OTF, 32 rows of 16 swizzled 16-byte chunks
constexpr int TC_WDESC_OFF = TC_B_BYTES + TC_GROUPS * TC_A_BYTES;
constexpr int TC_MISC_OFF = TC_WDESC_OFF + 640;  // >= TC_MAX_WFS * sizeof(WfsDev)
constexpr int TC_LOTF_OFF = TC_MISC_OFF + 128;
// dynamic shared memory of a launch caching nlotf uplink OTFs
__host__ __device__ constexpr int tc_smem_bytes(int nlotf) { return TC_LOTF_OFF + nlotf * TC_LOTF_BYTES; }
constexpr int TC_TMEM_COLS = 128 * TC_GROUPS;  // per group: 64 accumulator + 64 A operand
constexpr int TC_CTAS_PER_SM = 1;

// byte offset of (row r, 16-byte chunk c) in a K-major operand with kc chunks per row group
__host__ __device__ constexpr uint32_t tc_off(int r, int c, int kc) {
	return (uint32_t)(((r >> 3) * kc + c) * 128 + (r & 7) * 16);
}
// byte offset of (m-chunk mg, K-row k) in an MN-major operand with nkg k-groups
__host__ __device__ constexpr uint32_t mn_off(int mg, int k, int nkg) {
	return (uint32_t)((mg * nkg + (k >> 3)) * 128 + (k & 7) * 16);
}

struct TcTables {
	const uint4* bmat;  // TC_B_BYTES of B1|B2|B3|B4 images (bf16, canonical K-major layout)
};

// ---- PTX wrappers ----
__device__ __forceinline__ uint64_t globaltimer_ns() {
	uint64_t t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
	d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
	d |= (uint64_t)1 << 46;  // descriptor version for sm_100; SWIZZLE_NONE, base offset 0
	return d;
}
// kind::f16 instruction descriptor: D=F32, A=B=BF16, B K-major, M=128; A
// MN-major when a_mn (bit 15)
__host__ __device__ constexpr uint32_t tc_idesc(int n, bool a_mn) {
	return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? (1u << 15) : 0u) | ((uint32_t)(n >> 3) << 17) |
		   ((uint32_t)(128 >> 4) << 24);
}

// A from shared memory (descriptor)
__device__ __forceinline__ void tc_mma_ss(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
	asm volatile(
		"{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
		"l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
// A from tensor memory
__device__ __forceinline__ void tc_mma_ts(uint32_t dtmem, uint32_t atmem, uint64_t bd, uint32_t idesc, uint32_t acc) {
	asm volatile(
		"{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(dtmem),
		"r"(atmem), "l"(bd), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void tc_commit(uint64_t* mbar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
				 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void group_sync(int id) { asm volatile("barrier.sync %0, 128;" ::"r"(id) : "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
		: "=r"(ok)
		: "r"(smem_u32(m)), "r"(parity)
		: "memory");
	return ok != 0;
}

// 16 / 8 consecutive TMEM columns of this warp's 32 lanes <-> registers
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
	uint32_t r[16];
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
		  "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr));
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
	uint32_t r[8];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
				 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
				 : "r"(taddr));
#pragma unroll
	for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
	asm volatile(
		"tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
			taddr),
		"r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
		"r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
		: "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
	asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
				 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
				 : "memory");
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t (&r)[4]) {
	asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(r[0]), "r"(r[1]),
				 "r"(r[2]), "r"(r[3])
				 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Transfer-function factors of one quarter (8 spatial frequencies fy) of an
// OTF row, as complex pairs: (x, y) for fy, (z, w) for fy + 1.  l: uplink OTF
// (applied conjugated), e: ETF, or the real DTF nominal as (d, 0), or 1.
struct TfQuarter {
	float4 l[4], e[4];
};
__device__ __forceinline__ void tf_load(TfQuarter& t, const unsigned char* lrow_s, int swz, const float4* lrow,
	const float4* erow, const float2* nrow, int q) {
#pragma unroll
	for (int i = 0; i < 4; i++) {
		if (lrow_s)
			t.l[i] = *reinterpret_cast<const float4*>(lrow_s + (((4 * q + i) ^ swz) << 4));
		else
			t.l[i] = lrow ? __ldg(lrow + 4 * q + i) : make_float4(1.f, 0.f, 1.f, 0.f);
		if (erow) {
			t.e[i] = __ldg(erow + 4 * q + i);
		} else if (nrow) {
			const float2 d = __ldg(nrow + 4 * q + i);
			t.e[i] = make_float4(d.x, 0.f, d.y, 0.f);
		} else {
			t.e[i] = make_float4(1.f, 0.f, 1.f, 0.f);
		}
	}
}

// ---- operand split ----
// (a, b) -> packed bf16 pair hi = (bf16(a), bf16(b)) and lo = bf16 of the
// remainders; the first element sits in the low half.
__device__ __forceinline__ void split_pair(float a, float b, uint32_t& hi, uint32_t& lo) {
	const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
	const uint32_t hu = *reinterpret_cast<const uint32_t*>(&h);
	const float ha = __uint_as_float(hu << 16), hb = __uint_as_float(hu & 0xffff0000u);
	const __nv_bfloat162 l = __floats2bfloat162_rn(a - ha, b - hb);
	hi = hu;
	lo = *reinterpret_cast<const uint32_t*>(&l);
}
// 8 floats -> one 16-byte hi chunk and one lo chunk
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
	split_pair(x[0], x[1], hi.x, lo.x);
	split_pair(x[2], x[3], hi.y, lo.y);
	split_pair(x[4], x[5], hi.z, lo.z);
	split_pair(x[6], x[7], hi.w, lo.w);
}
__device__ __forceinline__ void sts128(unsigned char* base, uint32_t off, const uint4& v) {
	*reinterpret_cast<uint4*>(base + off) = v;
}

// sin(pi t), cos(pi t): t reduced exactly to [-1, 1] (t - 2 rint(t/2) is
// exact in FP32), then the hardware sine/cosine, whose absolute error on
// [-pi, pi] (about 4e-7) is far below the BF16x3 products' (about 1e-5).
__device__ __forceinline__ void sincospi_fast(float t, float& s, float& c) {
	const float r = fmaf(-2.f, rintf(0.5f * t), t);
	__sincosf(3.14159265358979f * r, &s, &c);
}

// ---- GEMM issue (one thread) ----
// D = sum_j Ah_j Bh_j + Ah_j Bl_j + Al_j Bh_j over nks K-steps of 16.  The
// descriptors are formed once per kernel; a K-step of 16 advances a start
// address by 256 B, i.e. the descriptor's start field by 16 (smem addresses
// are below 2^18, so the 14-bit field never carries).
// B: descriptor of its K-major image (SBO = chunks per row group x 128 B),
// lo half blo chunks further on.
// A in TMEM: hi K pairs in columns [acol, acol+alo), lo in [acol+alo, ...)
__device__ __forceinline__ void tc_gemm_ts(uint32_t dt, uint32_t acol, int alo, uint64_t bd, int blo, int nks,
	uint32_t idesc) {
	for (int j = 0; j < nks; j++) {
		const uint32_t ah = acol + 8 * j, al = acol + alo + 8 * j;
		const uint64_t bh = bd + (uint64_t)(16 * j), bl = bd + (uint64_t)(8 * blo + 16 * j);
		tc_mma_ts(dt, ah, bh, idesc, j > 0 ? 1u : 0u);
		tc_mma_ts(dt, ah, bl, idesc, 1u);
		tc_mma_ts(dt, al, bh, idesc, 1u);
	}
}
// A in shared memory, MN-major with nkg k-groups (descriptor ad, SBO = nkg x
// 128 B): hi K-rows from k-group 0, lo K-rows from k-group nkg/2
__device__ __forceinline__ void tc_gemm_ss(uint32_t dt, uint64_t ad, int nkg, uint64_t bd, int blo, int nks,
	uint32_t idesc) {
	for (int j = 0; j < nks; j++) {
		const uint64_t ah = ad + (uint64_t)(16 * j), al = ad + (uint64_t)(4 * nkg + 16 * j);
		const uint64_t bh = bd + (uint64_t)(16 * j), bl = bd + (uint64_t)(8 * blo + 16 * j);
		tc_mma_ss(dt, ah, bh, idesc, j > 0 ? 1u : 0u);
		tc_mma_ss(dt, ah, bl, idesc, 1u);
		tc_mma_ss(dt, al, bh, idesc, 1u);
	}
}

// ---------------------------------------------------------------------------
// Noise-free pixel intensities of nitem = nsa x nw subaperture images (item
// i -> subaperture i / nw of WFS i % nw, nw <= TC_MAX_WFS) into wfs[].ints;
// photon/read noise and gradients follow in noise_grad_kernel.  nlotf: 0, or
// nw when every WFS of the launch has an uplink OTF, which is then cached in
// shared memory.
__global__ void __launch_bounds__(TC_THREADS, TC_CTAS_PER_SM) ints_tc_kernel(PowfsDev P,
	const WfsDev* __restrict__ wfs, int nw, int nitem, int nlotf, TcTables T, int* errflag) {
	static_assert(TC_MAX_WFS * sizeof(WfsDev) <= 640, "WFS descriptor area");
	extern __shared__ __align__(128) unsigned char smem[];
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int g = warp >> 2, wq = warp & 3;  // tile group, warp within the group
	unsigned char* bbuf = smem;               // B1 | B2 | B3 | B4
	unsigned char* abuf = smem + TC_B_BYTES + g * TC_A_BYTES;
	WfsDev* wsm = reinterpret_cast<WfsDev*>(smem + TC_WDESC_OFF);
	const unsigned char* lotf_s = smem + TC_LOTF_OFF;
	uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + TC_MISC_OFF) + g;
	uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + TC_MISC_OFF + 32);
	int* bail = reinterpret_cast<int*>(smem + TC_MISC_OFF + 64) + g;

	for (int i = tid; i < TC_B_BYTES / 16; i += TC_THREADS) reinterpret_cast<uint4*>(bbuf)[i] = T.bmat[i];
	for (int i = tid; i < nw * (int)(sizeof(WfsDev) / 4); i += TC_THREADS)
		reinterpret_cast<uint32_t*>(wsm)[i] = reinterpret_cast<const uint32_t*>(wfs)[i];
	// uplink OTFs: row fx holds 16 chunks of 2 complex values, chunk c stored
	// at c ^ (fx & 15) so that the 32 rows read by a warp hit distinct banks
	for (int k = 0; k < nlotf; k++) {
		const uint4* src = reinterpret_cast<const uint4*>(wfs[k].lotfT);
		for (int i = tid; i < 512; i += TC_THREADS) {
			const int fx = i >> 4, c = i & 15;
			*reinterpret_cast<uint4*>(smem + TC_LOTF_OFF + k * TC_LOTF_BYTES + fx * 256 + ((c ^ (fx & 15)) << 4)) =
				src[i];
		}
	}
	if (tid == 0) {
		for (int k = 0; k < TC_GROUPS; k++) {
			mbar_init(reinterpret_cast<uint64_t*>(smem + TC_MISC_OFF) + k, 1);
			reinterpret_cast<int*>(smem + TC_MISC_OFF + 64)[k] = 0;
		}
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
					 "r"(TC_TMEM_COLS));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	fence_async_smem();
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tslot;
	const uint32_t dcol = tmem + 128 * g;  // accumulator columns of this group (lane 0)
	const uint32_t acol = dcol + 64;       // A-operand columns of this group
	const uint32_t tl = (uint32_t)(32 * wq) << 16;  // this warp's lane quarter
	const uint32_t a_s = smem_u32(abuf), b1_s = smem_u32(bbuf), b2_s = b1_s + TC_B1_BYTES,
				   b3_s = b2_s + TC_B2_BYTES, b4_s = b3_s + TC_B3_BYTES;
	const uint64_t bd1 = tc_desc(b1_s, 128, 8 * 128), bd2 = tc_desc(b2_s, 128, 16 * 128),
				   bd3 = tc_desc(b3_s, 128, 16 * 128), bd4 = tc_desc(b4_s, 128, 16 * 128);
	const uint64_t ad8 = tc_desc(a_s, 128, 8 * 128), ad16 = tc_desc(a_s, 128, 16 * 128);
	const bool issuer = (tid & 127) == 0;
	const int bar_id = 1 + g;
	uint32_t phase = 0;

	// operands written (tcgen05.st waited / generic smem fenced by the caller)
	// -> one thread issues and waits -> the group proceeds with the result
	auto finish_stage = [&](auto issue) -> bool {
		tc_fence_before();
		group_sync(bar_id);
		if (issuer) {
			tc_fence_after();
			issue();
			tc_commit(mbar);
			const uint64_t t0 = globaltimer_ns();
			while (!mbar_try_wait(mbar, phase)) {
				if (globaltimer_ns() - t0 > 2000000000ull) {
					atomicExch(errflag, SHWFS_ETIMEOUT_CODE);
					*bail = 1;
					break;
				}
			}
		}
		phase ^= 1u;
		group_sync(bar_id);
		tc_fence_after();
		return *bail == 0;
	};

	const int ntile = (nitem + 3) / 4;
	for (int t = TC_GROUPS * blockIdx.x + g; t < ntile; t += TC_GROUPS * gridDim.x) {
		const int item = 4 * t + wq;
		const bool valid = item < nitem;
		const int isa = valid ? item / nw : 0;
		const int iw = valid ? item % nw : 0;
		const WfsDev& W = wsm[iw];
		// the ETF row this lane multiplies at 4b -> 6a, fetched into L2 now
		if (valid && P.etfT1) {
			const float2* e = P.etfT1 + (size_t)isa * 1024 + 32 * lane;
			prefetch_l2(e);
			prefetch_l2(e + 16);
			if (P.etfT2) {
				prefetch_l2(P.etfT2 + (size_t)isa * 1024 + 32 * lane);
				prefetch_l2(P.etfT2 + (size_t)isa * 1024 + 32 * lane + 16);
			}
		}
		if (valid && W.grad && W.mtche && 32 * lane < 2 * P.npix) prefetch_l2(W.mtche + (size_t)isa * 2 * P.npix + 32 * lane);
		// ---- (b) field -> A(2a) in TMEM: row x = lane holds E(x-8, y), zero outside [8,24)
		{
			const int xp = lane - 8;
			const bool live = valid && xp >= 0 && xp < 16;
			const size_t base = (size_t)isa * 256 + (live ? xp : 0);
			float o[16], a[16];
			float s = 0.f;
#pragma unroll
			for (int y = 0; y < 16; y++) {
				o[y] = live ? __ldg(W.opd + base + y * 16) : 0.f;
				a[y] = live ? __ldg(W.amp + base + y * 16) : 0.f;
				s += o[y];
			}
#pragma unroll
			for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
			const float piston = s * (1.f / 256.f);
			uint32_t hw[16], lw[16];
#pragma unroll
			for (int y = 0; y < 16; y += 2) {
				float s0, c0, s1, c1;
				sincospi_fast(P.twoinvwvl * (o[y] - piston), s0, c0);
				sincospi_fast(P.twoinvwvl * (o[y + 1] - piston), s1, c1);
				split_pair(a[y] * c0, a[y + 1] * c1, hw[y / 2], lw[y / 2]);          // re: K = y
				split_pair(a[y] * s0, a[y + 1] * s1, hw[8 + y / 2], lw[8 + y / 2]);  // im: K = 16 + y
			}
			tmem_st16(acol + tl, hw);
			tmem_st16(acol + tl + 16, lw);
			tmem_wait_st();
		}
		if (!finish_stage([&] { tc_gemm_ts(dcol, acol, 16, bd1, 4, 2, tc_idesc(64, false)); })) break;  // 2a
		// ---- 2a out: row x holds F1(x-8, ky) -> K-rows x-8 (re), 16+x-8 (im) of A(2b), M = (s, ky)
		{
			const int xp = lane - 8;
			const bool live = xp >= 0 && xp < 16;
#pragma unroll
			for (int h = 0; h < 2; h++) {
				float re[16], im[16];
				tmem_ld16(dcol + tl + 16 * h, re);
				tmem_ld16(dcol + tl + 32 + 16 * h, im);
				tmem_wait_ld();
#pragma unroll
				for (int c = 0; c < 2; c++) {
					const int mg = 4 * wq + 2 * h + c;
					uint4 rh, rl, ih, il;
					split8(re + 8 * c, rh, rl);
					split8(im + 8 * c, ih, il);
					if (live) {
						sts128(abuf, mn_off(mg, xp, 8), rh);
						sts128(abuf, mn_off(mg, 16 + xp, 8), ih);
						sts128(abuf, mn_off(mg, 32 + xp, 8), rl);
						sts128(abuf, mn_off(mg, 48 + xp, 8), il);
					}
				}
			}
			fence_async_smem();
		}
		if (!finish_stage([&] { tc_gemm_ss(dcol, ad8, 8, bd1, 4, 2, tc_idesc(64, true)); })) break;  // 2b
		// ---- 2b out: row ky holds F(kx, ky) -> P = |F|^2 -> A(4a) in TMEM, K = kx
		{
			uint32_t hw[16], lw[16];
#pragma unroll
			for (int h = 0; h < 2; h++) {
				float re[16], im[16];
				tmem_ld16(dcol + tl + 16 * h, re);
				tmem_ld16(dcol + tl + 32 + 16 * h, im);
				tmem_wait_ld();
#pragma unroll
				for (int i = 0; i < 16; i += 2) {
					const float p0 = fmaf(re[i], re[i], im[i] * im[i]);
					const float p1 = fmaf(re[i + 1], re[i + 1], im[i + 1] * im[i + 1]);
					split_pair(p0, p1, hw[8 * h + i / 2], lw[8 * h + i / 2]);
				}
			}
			tmem_st16(acol + tl, hw);
			tmem_st16(acol + tl + 16, lw);
			tmem_wait_st();
		}
		if (!finish_stage([&] { tc_gemm_ts(dcol, acol, 16, bd2, 8, 2, tc_idesc(64, false)); })) break;  // 4a
		// ---- 4a out: row ky holds Q(ky, fx) -> K-rows ky (re), 32+ky (im) of A(4b), M = (s, fx)
		{
#pragma unroll
			for (int h = 0; h < 2; h++) {
				float re[16], im[16];
				tmem_ld16(dcol + tl + 16 * h, re);
				tmem_ld16(dcol + tl + 32 + 16 * h, im);
				tmem_wait_ld();
#pragma unroll
				for (int c = 0; c < 2; c++) {
					const int mg = 4 * wq + 2 * h + c;
					uint4 rh, rl, ih, il;
					split8(re + 8 * c, rh, rl);
					split8(im + 8 * c, ih, il);
					sts128(abuf, mn_off(mg, lane, 16), rh);
					sts128(abuf, mn_off(mg, 32 + lane, 16), ih);
					sts128(abuf, mn_off(mg, 64 + lane, 16), rl);
					sts128(abuf, mn_off(mg, 96 + lane, 16), il);
				}
			}
			fence_async_smem();
		}
		// the transfer function of 4b -> 6a in quarters of 8 fy: the loads of
		// quarter 0 are in flight during the 4b GEMM, those of quarter q+1
		// during the arithmetic of quarter q
		const unsigned char* lrow_s = (valid && nlotf) ? lotf_s + iw * TC_LOTF_BYTES + lane * 256 : nullptr;
		const float4* lrow =
			(valid && !nlotf && W.lotfT) ? reinterpret_cast<const float4*>(W.lotfT + 32 * lane) : nullptr;
		const float4* erow =
			(valid && P.etfT1) ? reinterpret_cast<const float4*>(P.etfT1 + (size_t)isa * 1024 + 32 * lane) : nullptr;
		const float4* erow2 =
			(erow && P.etfT2) ? reinterpret_cast<const float4*>(P.etfT2 + (size_t)isa * 1024 + 32 * lane) : nullptr;
		const float2* nrow = (valid && !P.etfT1 && P.nominalT)
								 ? reinterpret_cast<const float2*>(
									   P.nominalT + (P.nominal_per_sa ? (size_t)isa * 1024 : 0) + 32 * lane)
								 : nullptr;
		TfQuarter tq;
		tf_load(tq, lrow_s, lane & 15, lrow, erow, nrow, 0);
		if (!finish_stage([&] { tc_gemm_ss(dcol, ad16, 16, bd2, 8, 4, tc_idesc(64, true)); })) break;  // 4b
		// ---- 4b out: row fx holds OTF(fx, fy) x conj(uplink) x ETF -> A(6a) in TMEM, K = fy
		{
#pragma unroll
			for (int q = 0; q < 4; q++) {
				float re[8], im[8];
				tmem_ld8(dcol + tl + 8 * q, re);
				tmem_ld8(dcol + tl + 32 + 8 * q, im);
				TfQuarter tn;
				if (q < 3) tf_load(tn, lrow_s, lane & 15, lrow, erow, nrow, q + 1);
				tmem_wait_ld();
#pragma unroll
				for (int i = 0; i < 4; i++) {
					const float4 l = tq.l[i];
					float4 e = tq.e[i];
					if (erow2) {  // ETF interpolated between two sodium profiles
						const float4 e2 = __ldg(erow2 + 4 * q + i);
						e = make_float4(e.x * P.etfwt1 + e2.x * P.etfwt2, e.y * P.etfwt1 + e2.y * P.etfwt2,
							e.z * P.etfwt1 + e2.z * P.etfwt2, e.w * P.etfwt1 + e2.w * P.etfwt2);
					}
					float a = re[2 * i], b = im[2 * i];
					float a1 = fmaf(a, l.x, b * l.y), b1 = fmaf(b, l.x, -a * l.y);
					re[2 * i] = fmaf(a1, e.x, -b1 * e.y);
					im[2 * i] = fmaf(a1, e.y, b1 * e.x);
					a = re[2 * i + 1];
					b = im[2 * i + 1];
					a1 = fmaf(a, l.z, b * l.w);
					b1 = fmaf(b, l.z, -a * l.w);
					re[2 * i + 1] = fmaf(a1, e.z, -b1 * e.w);
					im[2 * i + 1] = fmaf(a1, e.w, b1 * e.z);
				}
				uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
				for (int i = 0; i < 4; i++) {
					split_pair(re[2 * i], re[2 * i + 1], rh[i], rl[i]);
					split_pair(im[2 * i], im[2 * i + 1], ih[i], il[i]);
				}
				tmem_st4(acol + tl + 4 * q, rh);       // re fy: K 0..31  -> hi columns 0..15
				tmem_st4(acol + tl + 16 + 4 * q, ih);  // im fy: K 32..63 -> hi columns 16..31
				tmem_st4(acol + tl + 32 + 4 * q, rl);  // lo columns 32..63
				tmem_st4(acol + tl + 48 + 4 * q, il);
				if (q < 3) tq = tn;
			}
			tmem_wait_st();
		}
		if (!finish_stage([&] { tc_gemm_ts(dcol, acol, 32, bd3, 8, 4, tc_idesc(32, false)); })) break;  // 6a
		// ---- 6a out: row fx holds T(fx, iy) -> K-rows fx (re), 32+fx (im) of A(6b), M = (s, iy < 8)
		{
			float re[8], im[8];
			tmem_ld8(dcol + tl, re);
			tmem_ld8(dcol + tl + 16, im);
			tmem_wait_ld();
			uint4 rh, rl, ih, il;
			split8(re, rh, rl);
			split8(im, ih, il);
			const int mg = 4 * wq;
			sts128(abuf, mn_off(mg, lane, 16), rh);
			sts128(abuf, mn_off(mg, 32 + lane, 16), ih);
			sts128(abuf, mn_off(mg, 64 + lane, 16), rl);
			sts128(abuf, mn_off(mg, 96 + lane, 16), il);
			fence_async_smem();
		}
		if (!finish_stage([&] { tc_gemm_ss(dcol, ad16, 16, bd4, 8, 4, tc_idesc(16, true)); })) break;  // 6b
		// ---- 6b out: row iy (lanes 0..7) holds I(ix, iy) -> noise-free pixels of this warp's subaperture
		{
			float v[8];
			tmem_ld8(dcol + tl, v);
			tmem_wait_ld();
			const int npx = P.pixpsax, npy = P.pixpsay;
			if (valid && W.ints && lane < npy) {
				float* o = W.ints + (size_t)isa * P.npix + lane * npx;
				const float alpha = W.alpha;
#pragma unroll
				for (int ix = 0; ix < 8; ix++)
					if (ix < npx) o[ix] = P.accum ? o[ix] + v[ix] * alpha : v[ix] * alpha;
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

}  // namespace shwfs
