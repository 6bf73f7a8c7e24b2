// Tensor-core (tcgen05) form of the imaging stages (b)-(e), n_opd=16, n_f=32.
//
// Every transform of the subaperture chain is a real GEMM on the 5th-gen
// tensor cores with BF16 operands split in three terms (a*b ~ ah*bh + ah*bl +
// al*bh, x = xh + xl, xl = bf16(x - xh)) and FP32 accumulators in TMEM:
//
//   2a  F1(x, ky)  = sum_y  E(x, y)  w32^(ky(y+8))     rows (s, x),  K = y
//   2b  F(kx, ky)  = sum_x  F1(x,ky) w32^(kx(x+8))     rows (s, ky), K = x
//   4a  Q(ky, fx)  = sum_kx P(kx,ky) w32^(fx kx)       rows (s, ky), K = kx  (P = |F|^2)
//   4b  O(fx, fy)  = sum_ky Q(ky,fx) w32^(fy ky)       rows (s, fx), K = ky
//   6a  T(fx, iy)  = sum_fy O'(fx,fy) Gy(iy, fy)       rows (s, fx), K = fy  (O' = O x conj(uplink) x ETF)
//                                                       N = 32: Re iy in columns 0..15, Im in 16..31
//   6b  I(ix, iy)  = Re sum_fx Gx(ix, fx) T(fx, iy)    FP32 warp reduction
//
// with w32 = exp(-2 pi i / 32) (FFTW's forward sign) and G = the inverse DFT
// premultiplied by the separable bilinear pixel weights, so the inverse
// transform and the pixel sampling of maos/wfsints.c:284-286 collapse into
// 6a/6b.  A tile is 4 subapertures = 128 GEMM rows; warp w owns subaperture w
// of the tile and TMEM lanes 32w..32w+31.  One elected thread issues the MMAs
// and commits them to an mbarrier that every thread waits on (bounded wait:
// on expiry the kernel records SHWFS_ETIMEOUT, frees its TMEM and returns).
//
// Shared memory per CTA: a 32 KB operand region (warp w's 8 KB slice holds its
// 32 A-rows, and doubles as its FP32 transpose tile between stages) and the
// 32 KB of constant B operands.  Operands use the K-major, no-swizzle
// canonical layout: core matrices of 8 rows x 16 bytes, 128 bytes apart
// along K (LBO) and 16 x 128 bytes apart along rows (SBO).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "shwfs_kernels.cuh"

namespace shwfs {

constexpr int SHWFS_ETIMEOUT_CODE = -5;  // SHWFS_ETIMEOUT of shwfs_b200.h

// ---- constants of the operand layouts ----
constexpr int TC_A_BYTES = 128 * 16 * 16;  // 128 rows x 16 chunks x 16 B
constexpr int TC_B1_BYTES = 64 * 8 * 16;   // N=64, K=32 (h|l: 8 chunks)
constexpr int TC_B2_BYTES = 64 * 16 * 16;  // N=64, K=64 (h|l: 16 chunks)
constexpr int TC_B3_BYTES = 32 * 16 * 16;  // N=32 (16 re + 16 im pixel rows), K=64
constexpr int TC_B_BYTES = TC_B1_BYTES + TC_B2_BYTES + TC_B3_BYTES;
constexpr int TC_SMEM_BYTES = TC_A_BYTES + TC_B_BYTES + 64;
constexpr int TC_TMEM_COLS = 64;

// byte offset of (row r, 16-byte chunk c) in an operand with kc chunks per row group
__host__ __device__ constexpr uint32_t tc_off(int r, int c, int kc) {
	return (uint32_t)(((r >> 3) * kc + c) * 128 + (r & 7) * 16);
}

struct TcTables {
	const uint4* bmat;  // TC_B_BYTES of B1|B2|B3 images (bf16, canonical layout)
	const float2* gx;   // pixpsax x 32 : Gx(ix, fx)
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
// kind::f16 instruction descriptor: D=F32, A=B=BF16, both K-major, M=128
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
	return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
	asm volatile(
		"{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
		"l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void tc_commit(uint64_t* mbar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
				 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

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

// 16 consecutive TMEM columns of this warp's 32 lanes -> 16 registers per thread
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
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- operand writers ----
// bf16 hi/lo split of 8 floats packed as two 16-byte chunks
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
	uint32_t h[4], l[4];
#pragma unroll
	for (int i = 0; i < 4; i++) {
		const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * i]), h1 = __float2bfloat16_rn(x[2 * i + 1]);
		const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * i] - __bfloat162float(h0));
		const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * i + 1] - __bfloat162float(h1));
		h[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
		l[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
	}
	hi = make_uint4(h[0], h[1], h[2], h[3]);
	lo = make_uint4(l[0], l[1], l[2], l[3]);
}
// Writes row r of the A operand from K real values x[0..K): hi chunks 0..K/8-1,
// lo chunks 8..8+K/8-1 (K = 32 or 64).
template <int K>
__device__ __forceinline__ void write_arow(unsigned char* abuf, int r, const float* x) {
#pragma unroll
	for (int c = 0; c < K / 8; c++) {
		uint4 hi, lo;
		split8(x + 8 * c, hi, lo);
		*reinterpret_cast<uint4*>(abuf + tc_off(r, c, 16)) = hi;
		*reinterpret_cast<uint4*>(abuf + tc_off(r, 8 + c, 16)) = lo;
	}
}

// Issues the 3-term split product over nks K-steps (16 real K each):
// D = sum_j Ah_j Bh_j + Ah_j Bl_j + Al_j Bh_j.  bbase: B image, bkc: its
// chunks per row group, blo: chunk index of its lo half.
__device__ __forceinline__ void tc_gemm(uint32_t dtmem, uint32_t abase, uint32_t bbase, int bkc, int blo, int nks,
	uint32_t idesc) {
	const uint32_t asbo = 16 * 128, bsbo = (uint32_t)bkc * 128;
	uint32_t acc = 0;
	for (int j = 0; j < nks; j++) {
		const uint64_t ah = tc_desc(abase + (2 * j) * 128, 128, asbo);
		const uint64_t al = tc_desc(abase + (8 + 2 * j) * 128, 128, asbo);
		const uint64_t bh = tc_desc(bbase + (2 * j) * 128, 128, bsbo);
		const uint64_t bl = tc_desc(bbase + (blo + 2 * j) * 128, 128, bsbo);
		tc_mma(dtmem, ah, bh, idesc, acc);
		acc = 1;
		tc_mma(dtmem, ah, bl, idesc, 1);
		tc_mma(dtmem, al, bh, idesc, 1);
	}
}

// FP32 transpose tile of one warp: 32 x 32 float2 with an XOR swizzle so that
// both row and column accesses are bank-conflict free.
__device__ __forceinline__ float2* tile_at(float2* t, int row, int col) { return t + row * 32 + (col ^ row); }

// ---------------------------------------------------------------------------
template <int NPQ>
__global__ void __launch_bounds__(128) ints_tc_kernel(PowfsDev P, const WfsDev* __restrict__ wfs, int nw, int nitem,
	TcTables T, int* errflag) {
	extern __shared__ __align__(128) unsigned char smem[];
	unsigned char* abuf = smem;                        // 32 KB: A operands / transpose tiles
	unsigned char* bbuf = smem + TC_A_BYTES;           // 28 KB: B1 | B2 | B3
	uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + TC_A_BYTES + TC_B_BYTES);
	uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + TC_A_BYTES + TC_B_BYTES + 8);
	int* bail = reinterpret_cast<int*>(smem + TC_A_BYTES + TC_B_BYTES + 16);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

	// constant B operands into shared memory
	for (int i = tid; i < TC_B_BYTES / 16; i += 128) reinterpret_cast<uint4*>(bbuf)[i] = T.bmat[i];
	if (tid == 0) {
		mbar_init(mbar, 1);
		*bail = 0;
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
	const uint32_t tlane = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's lanes
	const uint32_t a_s = smem_u32(abuf), b1_s = smem_u32(bbuf), b2_s = b1_s + TC_B1_BYTES,
				   b3_s = b2_s + TC_B2_BYTES;
	unsigned char* myslice = abuf + warp * 8192;  // rows 32*warp.. of the A operand
	float2* tile = reinterpret_cast<float2*>(myslice);
	uint32_t phase = 0;

	// one MMA stage: operands written -> issue -> wait
	auto run_stage = [&](uint32_t bbase, int bkc, int blo, int nks, int n) -> bool {
		fence_async_smem();
		tc_fence_before();
		__syncthreads();
		if (tid == 0) {
			tc_fence_after();
			tc_gemm(tmem, a_s, bbase, bkc, blo, nks, tc_idesc(n));
			tc_commit(mbar);
		}
		// bounded wait: 2 s of wall time, then record the expiry and leave
		const uint64_t t0 = globaltimer_ns();
		while (!mbar_try_wait(mbar, phase)) {
			if (globaltimer_ns() - t0 > 2000000000ull) {
				atomicExch(errflag, SHWFS_ETIMEOUT_CODE);
				*bail = 1;
				break;
			}
		}
		phase ^= 1u;
		tc_fence_after();
		return *bail == 0;
	};

	const int ntile = (nitem + 3) / 4;
	for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
		const int item = 4 * t + warp;
		const bool valid = item < nitem;
		const int isa = valid ? item / nw : 0;
		const WfsDev W = wfs[valid ? item % nw : 0];
		// ---- (b) field: row x = lane holds E(x-8, y) for x in [8,24), else 0
		{
			const float* opd = W.opd + (size_t)isa * 256;
			const float* amp = W.amp + (size_t)isa * 256;
			const int xp = lane - 8;
			const bool live = valid && xp >= 0 && xp < 16;
			float o[16], a[16];
			float s = 0.f;
#pragma unroll
			for (int y = 0; y < 16; y++) {
				o[y] = live ? __ldg(opd + y * 16 + xp) : 0.f;
				a[y] = live ? __ldg(amp + y * 16 + xp) : 0.f;
				s += o[y];
			}
#pragma unroll
			for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
			const float piston = s * (1.f / 256.f);
			float row[32];
#pragma unroll
			for (int y = 0; y < 16; y++) {
				float sn, cs;
				sincospif(P.twoinvwvl * (o[y] - piston), &sn, &cs);
				row[y] = live ? a[y] * cs : 0.f;
				row[16 + y] = live ? a[y] * sn : 0.f;
			}
			write_arow<32>(abuf, 32 * warp + lane, row);
		}
		if (!run_stage(b1_s, 8, 4, 2, 64)) break;  // 2a
		// ---- 2a out (row x) -> transpose -> 2b in (row ky), K = x-8
		{
			float v[16];
#pragma unroll
			for (int q = 0; q < 4; q++) {  // columns 16q..16q+15: re ky 0..31 then im
				tmem_ld16(tlane + 16 * q, v);
				tmem_wait_ld();
				if (lane >= 8 && lane < 24) {
#pragma unroll
					for (int i = 0; i < 16; i++) {
						const int c = 16 * q + i, ky = c & 31;
						float2* e = tile_at(tile, ky, lane - 8);
						if (c < 32) e->x = v[i];
						else e->y = v[i];
					}
				}
			}
			__syncwarp();
			float row[32];
#pragma unroll
			for (int xp = 0; xp < 16; xp++) {
				const float2 e = *tile_at(tile, lane, xp);
				row[xp] = e.x;
				row[16 + xp] = e.y;
			}
			__syncwarp();
			write_arow<32>(abuf, 32 * warp + lane, row);
		}
		if (!run_stage(b1_s, 8, 4, 2, 64)) break;  // 2b
		// ---- 2b out (row ky: F(kx, ky)) -> |F|^2 -> 4a in (row ky), K = kx
		{
			float re[16], im[16], row[32];
#pragma unroll
			for (int h = 0; h < 2; h++) {
				tmem_ld16(tlane + 16 * h, re);
				tmem_ld16(tlane + 32 + 16 * h, im);
				tmem_wait_ld();
#pragma unroll
				for (int i = 0; i < 16; i++) row[16 * h + i] = re[i] * re[i] + im[i] * im[i];
			}
			write_arow<32>(abuf, 32 * warp + lane, row);
		}
		if (!run_stage(b2_s, 16, 8, 2, 64)) break;  // 4a (real K: first half of B2)
		// ---- 4a out (row ky: Q(ky, fx)) -> transpose -> 4b in (row fx), K = ky (complex)
		{
			float v[16];
#pragma unroll
			for (int q = 0; q < 4; q++) {
				tmem_ld16(tlane + 16 * q, v);
				tmem_wait_ld();
#pragma unroll
				for (int i = 0; i < 16; i++) {
					const int c = 16 * q + i, fx = c & 31;
					float2* e = tile_at(tile, fx, lane);
					if (c < 32) e->x = v[i];
					else e->y = v[i];
				}
			}
			__syncwarp();
			float row[64];
#pragma unroll
			for (int ky = 0; ky < 32; ky++) {
				const float2 e = *tile_at(tile, lane, ky);
				row[ky] = e.x;
				row[32 + ky] = e.y;
			}
			__syncwarp();
			write_arow<64>(abuf, 32 * warp + lane, row);
		}
		if (!run_stage(b2_s, 16, 8, 4, 64)) break;  // 4b
		// ---- 4b out (row fx: OTF(fx, fy)) x conj(uplink) x ETF -> 6a in (row fx), K = fy
		{
			float row[64];
			float re[16], im[16];
#pragma unroll
			for (int h = 0; h < 2; h++) {
				tmem_ld16(tlane + 16 * h, re);
				tmem_ld16(tlane + 32 + 16 * h, im);
				tmem_wait_ld();
#pragma unroll
				for (int i = 0; i < 16; i++) {
					row[16 * h + i] = re[i];
					row[32 + 16 * h + i] = im[i];
				}
			}
			const int fx = lane;
			if (valid) {
				if (W.lotfT) {
					const float2* l = W.lotfT + 32 * fx;
#pragma unroll
					for (int fy = 0; fy < 32; fy++) {
						const float2 c = __ldg(l + fy);
						const float a = row[fy], b = row[32 + fy];
						row[fy] = fmaf(a, c.x, b * c.y);
						row[32 + fy] = fmaf(b, c.x, -a * c.y);
					}
				}
				if (P.etfT1) {
					const float2* e1 = P.etfT1 + (size_t)isa * 1024 + 32 * fx;
#pragma unroll
					for (int fy = 0; fy < 32; fy++) {
						float2 c = __ldg(e1 + fy);
						if (P.etfT2) {
							const float2 c2 = __ldg(P.etfT2 + (size_t)isa * 1024 + 32 * fx + fy);
							c = make_float2(c.x * P.etfwt1 + c2.x * P.etfwt2, c.y * P.etfwt1 + c2.y * P.etfwt2);
						}
						const float a = row[fy], b = row[32 + fy];
						row[fy] = fmaf(a, c.x, -b * c.y);
						row[32 + fy] = fmaf(a, c.y, b * c.x);
					}
				} else if (P.nominalT) {
					const float* nm = P.nominalT + (P.nominal_per_sa ? (size_t)isa * 1024 : 0) + 32 * fx;
#pragma unroll
					for (int fy = 0; fy < 32; fy++) {
						const float d = __ldg(nm + fy);
						row[fy] *= d;
						row[32 + fy] *= d;
					}
				}
			}
			write_arow<64>(abuf, 32 * warp + lane, row);
		}
		if (!run_stage(b3_s, 16, 8, 4, 32)) break;  // 6a
		// ---- 6a out (row fx: T(fx, iy)) -> 6b: I(ix,iy) = Re sum_fx Gx(ix,fx) T(fx,iy)
		float pix[NPQ];
		{
			float v[32];  // cols 0..15 re iy, 16..31 im iy
			{
				float a[16], b[16];
				tmem_ld16(tlane, a);
				tmem_ld16(tlane + 16, b);
				tmem_wait_ld();
#pragma unroll
				for (int i = 0; i < 16; i++) {
					v[i] = a[i];
					v[16 + i] = b[i];
				}
			}
			const int npx = P.pixpsax, npy = P.pixpsay, npix = P.npix;
			float* red = reinterpret_cast<float*>(myslice);  // [32 lanes][npix] partial sums
#pragma unroll 1
			for (int ix = 0; ix < npx; ix++) {
				const float2 g = __ldg(T.gx + ix * 32 + lane);
#pragma unroll
				for (int iy = 0; iy < 16; iy++) {
					if (iy < npy) red[lane * npix + ix + iy * npx] = fmaf(g.x, v[iy], -g.y * v[16 + iy]);
				}
			}
			__syncwarp();
#pragma unroll
			for (int q = 0; q < NPQ; q++) {
				const int p = lane + 32 * q;
				float sum = 0.f;
				if (p < npix) {
					for (int f = 0; f < 32; f++) sum += red[f * npix + p];
				}
				pix[q] = p < npix ? sum * W.alpha : 0.f;
			}
			__syncwarp();
		}
		if (valid) {
			const int npix = P.npix;
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
				grad_from_pixels<NPQ>(pix, npix, P.pixpsax, P.pixpsay, P, W.mtche + (size_t)isa * 2 * npix, W.i0sum,
					isa, lane, W.grad, P.nsa);
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

}  // namespace shwfs
