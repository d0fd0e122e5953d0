// K5: the modal sum P(z_j, r_n) = C(r_n) sum_m A_jm e^{i k_m r_n} as a dense
// complex contraction on the tcgen05 tensor cores
// (ModeSolver::getTLoss2D, ModeSolver.cpp:492-565, at many receivers).
//
//   A_jm = v_m(z_s) v_m(z_j) / sqrt(k_m)      (complex, receivers x modes)
//   E_mn = e^{i k_m r_n},  r_n = (n + 1) dr    (complex, modes x ranges)
//   C(r) = 1000 * 4 pi i e^{-i pi/4} / sqrt(8 pi r)
//
// As one real GEMM per group of 64 receivers:
//   D[128 x N] = A'[128 x 2M] * B'[2M x N],
//   A' = [[Re A, -Im A], [Im A, Re A]] (rows 0..63 give Re P, 64..127 Im P),
//   B' = [[Re E], [Im E]] interleaved per mode (k = 2m: Re, 2m + 1: Im).
// Three operand formats (template parameter F of the kernels):
//  * kMsBf16x3: each operand is split into bf16 hi + lo parts and D
//    accumulates A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32 (3-term
//    split-BF16, ~2^-16 relative per product; kind::f16, K = 16 per MMA);
//  * kMsTf32: each operand rounded to TF32 (10-bit mantissa, round to
//    nearest) and D accumulates A B in FP32 (one product, ~2^-11 relative;
//    kind::tf32, K = 8 per MMA);
//  * kMsBf16x6: each operand is split into bf16 hi + mid + lo parts (24
//    significant bits, an FP32 value exactly) and D accumulates the six
//    products hi hi, hi mid, mid hi, hi lo, mid mid, lo hi (the dropped ones
//    are ~2^-24 relative), so the result carries FP32-accumulation error only.
//    This is the guarded sum: the generators also add up |A'| per receiver
//    and tile, the finishing kernel flags every point whose |P| is too small
//    for that error to stay below 0.05 dB in TL, and k_ms_fix recomputes the
//    flagged points in FP64.
// A chunk's A' takes 16 KB (24 KB for kMsBf16x6) and its B' 32 KB (48 KB) of
// shared memory; the pipeline, barriers and epilogue are shared.
//
// Since r_n = r_n0 + o dr inside a 256-range tile (r_n0 its first range),
// E_mn = e^{i k_m r_n0} e^{i k_m o dr}: the tile's phase is folded into A
// (A'(tile) = A diag(e^{i k r_n0}), 64 x 16 complex products per chunk) and
// B' = e^{i k o dr} does not depend on the tile, so it is prepared once per
// chunk in FP64 and streamed in by TMA.  The tile phases are reduced mod 2 pi
// in FP64 before their cast to FP32.
//
// Persistent kernel: the (receiver group, 256-range tile, 16-mode chunk)
// units are split evenly over one CTA per SM; a CTA accumulates the chunks of
// one (group, tile) in TMEM (two accumulators, so a finished tile's epilogue
// overlaps the next tile's MMAs; the guarded sum restarts the accumulation
// every kMsAccChunks chunks and adds the blocks in the epilogue) and stores
// its partial sum of the tile in its own slot; the finishing kernel adds the
// slots of the CTAs that shared the tile.  Warp 0: TMEM allocation and
// tcgen05.mma issue.  Warp 9: bulk TMA of the chunk's B' image, A and tile
// phases into a 4-deep ring.  Warps 1-8: generate A'(tile) into a 3-deep
// ring of shared memory.  Warps 10-13: read the accumulators out (one TMEM
// lane quarter each), so that the generators never wait for an epilogue.
//
// Shared-memory operand layout: K-major, each operand row holds the 32 k of a
// chunk; bf16: 64 B rows, 64-byte swizzle, 8-row atoms of 512 B (sw64_off);
// TF32: 128 B rows, 128-byte swizzle, 8-row atoms of 1 KB (sw128_off).  The
// 16-byte chunks are XOR-permuted by row so that the generators' 16-byte
// stores and the tensor cores' reads are free of bank conflicts.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "device_common.cuh"

namespace ncpa {

namespace {

constexpr int kMsRows = 128;        // UMMA M (Re / Im rows of 64 receivers)
constexpr int kMsRcv = 64;          // receivers per group
constexpr int kMsNT = 256;          // ranges per tile (UMMA N)
constexpr int kMsModes = 16;        // modes per K-chunk
constexpr int kMsKC = 2 * kMsModes; // K per chunk
constexpr int kMsABytes = kMsRows * kMsKC * 2;   // one A' part (hi or lo) of a chunk: 8 KB
constexpr int kMsBBytes = kMsNT * kMsKC * 2;     // one B' part of a chunk: 16 KB
constexpr int kMsACBytes = kMsModes * kMsRcv * 8;  // a chunk's A as complex FP32, [mode][receiver]: 8 KB
constexpr int kMsQBytes = kMsModes * 8;            // tile phases of one chunk
constexpr int kMsGenWarps = 8;      // A' generators
constexpr int kMsGenThreads = 32 * kMsGenWarps;
constexpr int kMsProducerWarp = 1 + kMsGenWarps;  // warp 0: MMA issuer, 1-8: generators, 9: TMA producer
constexpr int kMsEpiWarp0 = kMsProducerWarp + 1;  // 10-13: epilogue (TMEM -> partial tiles)
constexpr int kMsEpiWarps = 4;
constexpr int kMsThreads = 32 * (kMsEpiWarp0 + kMsEpiWarps);
static_assert(kMsEpiWarps == 4 && kMsEpiWarp0 % 4 == 2, "one epilogue warp per TMEM lane quarter (warp % 4)");
constexpr int kEpiCols = 16;        // epilogue: accumulator columns per tcgen05.ld
constexpr int kEpiAhead = 4;        // column groups of old partial sums loaded ahead
constexpr int kMsAcc = 2;           // TMEM accumulators (kMsNT columns each): all 512 columns
constexpr int kMsMaxStages = 4;     // barrier arrays are sized for the deepest ring
static_assert(kMsAcc * kMsNT <= 512, "TMEM columns");
static_assert(kMsGenThreads == kMsRcv * (kMsModes / 4), "one generator per (receiver, mode quad)");

enum : int { kMsBf16x3 = 0, kMsTf32 = 1, kMsBf16x6 = 2 };

// guarded sum: the TL tolerance it keeps, and the bound eps of its error
// relative to S = sum_m |A'_jm| (the magnitude of the modal terms at the
// tile's first range): |P_tc - P| <= eps S.  The six-product split drops
// terms ~2^-24 relative, so the error is that of the FP32 accumulation in
// TMEM: each tcgen05.mma rounds the accumulator (12 per chunk), and the error
// grows with the accumulator's magnitude and the number of roundings.  So one
// accumulation covers at most kMsAccChunks chunks (64 modes) and the epilogue
// adds the blocks' partial tiles in FP32 (round to nearest).  kMsGuardEps is
// twice the largest |P_tc - P| / S measured over every point of a 1362-mode,
// 64-receiver x 20000-range sum (4.7e-7 with 12 block additions per CTA and
// tile; without blocks it was 2.2e-6, with 16-chunk blocks 1.3e-6); a CTA
// that adds more blocks than that calibration is charged 2^-24 S per extra
// addition (ms_guard_eps).  kMsAccChunks can be set at compile time for such
// calibration runs; kMsGuardEps holds for the default.
constexpr double kMsGuardTlDb = 0.05;
constexpr double kMsGuardEps = 1.0e-6;
constexpr long long kMsGuardCalAdds = 12;
#ifndef NCPA_MS_ACC_CHUNKS
#define NCPA_MS_ACC_CHUNKS 4
#endif
constexpr int kMsAccChunks = NCPA_MS_ACC_CHUNKS;

// shared-memory plan of a format: a TMA stage holds the chunk's B' image
// (kParts parts of 16 KB; TF32: one 32-bit image of the same size as two),
// A as complex FP32 and the tile phases (1 KB aligned); a generated A' stage
// holds kParts parts of 8 KB.  TS / GS: depths of the TMA and generated-A'
// rings (the schedule the autotuner picks among; the defaults are the
// deepest that fit).
template <int F, int TS = (F == kMsBf16x6 ? 3 : 4), int GS = (F == kMsBf16x6 ? 2 : 3)>
struct MsCfg {
    static constexpr int kParts = F == kMsBf16x6 ? 3 : 2;
    static constexpr int kBChunk = kParts * kMsBBytes;   // B' image bytes per chunk
    static constexpr int kOffAC = kBChunk;
    static constexpr int kOffQ = kOffAC + kMsACBytes;
    static constexpr int kTx = kBChunk + kMsACBytes + kMsQBytes;
    static constexpr int kTStageBytes = (kOffQ + kMsQBytes + 1023) / 1024 * 1024;
    static constexpr int kTStages = TS;
    static constexpr int kGStageBytes = kParts * kMsABytes;
    static constexpr int kGStages = GS;
    static constexpr int kOffGRing = kTStages * kTStageBytes;
    static constexpr int kSmem = kOffGRing + kGStages * kGStageBytes + 1024;
    static_assert(kSmem <= 232448 - 256, "shared memory per block");
    static_assert(kTStages <= kMsMaxStages && kGStages <= kMsMaxStages, "barrier arrays");
    static_assert(kMsACBytes % 16 == 0 && kMsQBytes % 16 == 0 && kTx % 16 == 0 && kBChunk % 1024 == 0 &&
                      kGStageBytes % 1024 == 0,
                  "bulk copies move 16-byte multiples; operand stages stay 1 KB aligned");
};

// byte offset of element (row, k) in a K-major tile of kMsKC = 32 bf16 per
// row with the 64-byte swizzle: rows of 64 B in atoms of 8 rows (512 B); the
// 16-byte chunk index k / 8 is XORed with (row / 2) % 4
__host__ __device__ __forceinline__ uint32_t sw64_off(int row, int k) {
    const int r = row & 7;
    return (uint32_t)((row >> 3) * 512 + r * 64 + ((((k >> 3) ^ (r >> 1)) & 3) << 4) + (k & 7) * 2);
}

// byte offset of element (row, k) in a K-major tile of kMsKC = 32 fp32 per
// row with the 128-byte swizzle: rows of 128 B in atoms of 8 rows (1 KB); the
// 16-byte chunk index k / 4 is XORed with row % 8
__host__ __device__ __forceinline__ uint32_t sw128_off(int row, int k) {
    const int r = row & 7;
    return (uint32_t)((row >> 3) * 1024 + r * 128 + ((((k >> 2) ^ r) & 7) << 4) + (k & 3) * 4);
}

// shared-memory matrix descriptor (tcgen05 format): start >> 4 in [0,14),
// leading-byte offset in [16,30) (unused by swizzled K-major layouts: 1),
// stride-byte offset >> 4 in [32,46) (next 8-row atom: 512 B), descriptor
// version 1 in [46,48), base offset 0, layout type 4 = 64-byte swizzle in
// [61,64).  A K-step of 16 elements advances the start address by 32 B.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
           (4ull << 61);
}
// same for the 128-byte swizzle: stride-byte offset 1 KB, layout type 2
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B bf16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 in [17,23),
// M >> 4 in [24,29)
constexpr uint32_t kMsIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMsNT >> 3) << 17) |
                              ((uint32_t)(kMsRows >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kMsIdesc), "r"(accumulate)
        : "memory");
}

// instruction descriptor, kind::tf32: FP32 accumulator, A and B TF32 (format
// 2 in bits 7-9 and 10-12), both K-major, same N and M
constexpr uint32_t kMsIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kMsNT >> 3) << 17) |
                                  ((uint32_t)(kMsRows >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kMsIdescTf32), "r"(accumulate)
        : "memory");
}

// fp32 -> tf32, round to nearest (ties away), as the 32-bit pattern the
// tensor cores read
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// hi / lo bf16 pairs of (re, im): lo keeps the next 8 bits of each value
__device__ __forceinline__ void split2(float2 v, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
    const __nv_bfloat162 l = __floats2bfloat162_rn(v.x - __low2float(h), v.y - __high2float(h));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// hi / mid / lo bf16 pairs of (re, im): 24 significant bits, so the three
// parts add up to the FP32 value (each remainder is exact in FP32)
__device__ __forceinline__ void split3(float2 v, uint32_t& hi, uint32_t& mid, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
    const float rx = v.x - __low2float(h), ry = v.y - __high2float(h);
    const __nv_bfloat162 m = __floats2bfloat162_rn(rx, ry);
    const __nv_bfloat162 l = __floats2bfloat162_rn(rx - __low2float(m), ry - __high2float(m));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    mid = *reinterpret_cast<const uint32_t*>(&m);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void sts128(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
                 : "memory");
}

}  // namespace

// ---------------------------------------------------------------------------
// preparation
// ---------------------------------------------------------------------------
// B' chunk images: B'[o][2m] = Re, B'[o][2m + 1] = Im of e^{i k_m o dr}
// (o = 0 .. 255, the range offset inside a tile; attenuation included unless
// lossless) in FP64, then split (bf16 hi, mid, lo or hi, lo) or rounded
// (TF32), in the shared-memory layout of the operand; zero for the padding
// modes m >= M.  The images do not depend on the tile: the tile's phase
// e^{i k r_n0} goes into A'.
//
// b64, when given, receives the same FP64 values as [o][M_pad] complex (the
// guarded sum's fix-up reads them).  A thread covers one range offset of four
// consecutive modes (a quad q4 of the chunk), so each operand part is one
// 16-byte chunk of the swizzled row (k = 8 q4 .. 8 q4 + 7: Re, Im of the four
// modes) written with one store.  Each value is evaluated directly (the
// phase k o dr reduced mod 2 pi in FP64, then sine / cosine and the
// attenuation factor): the threads are independent, so the launch spreads
// over every SM.
constexpr int kMsBQuads = kMsModes / 4;

__device__ __forceinline__ uint32_t bf16_pair(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

template <int F>
__device__ void ms_b_entry(long long id, int M, int M_pad, int n_chunks, const double* __restrict__ kr,
                           const double* __restrict__ ki, double dr, int lossless, unsigned char* __restrict__ img,
                           double2* __restrict__ b64) {
    const long long per_chunk = (long long)kMsNT * kMsBQuads;
    if (id >= (long long)n_chunks * per_chunk) return;
    const int o = (int)(id % kMsNT);
    const int q4 = (int)((id / kMsNT) % kMsBQuads);
    const int chunk = (int)(id / per_chunk);
    const int m0 = chunk * kMsModes + 4 * q4;
    const double x = (double)o * dr;
    double cr[4], ci[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        cr[v] = 0.0;
        ci[v] = 0.0;
        const int m = m0 + v;
        if (m < M) {
            const double th = kr[m] * x;
            const double red = fma(-rint(th * (0.5 / kPi)), 2.0 * kPi, th);
            double sn, cs;
            sincos(red, &sn, &cs);
            const double amp = lossless ? 1.0 : exp(-ki[m] * x);
            cr[v] = amp * cs;
            ci[v] = amp * sn;
        }
    }
    unsigned char* cimg = img + (size_t)chunk * MsCfg<F>::kBChunk;
    if (b64) {
        double2* row = b64 + (size_t)o * M_pad + m0;
#pragma unroll
        for (int v = 0; v < 4; ++v) row[v] = make_double2(cr[v], ci[v]);
    }
    if (F == kMsBf16x6) {
        // three bf16 parts of the FP64 value: hi, then the remainders
        uint32_t h[4], md[4], l[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const __nv_bfloat16 hr = __double2bfloat16(cr[v]), hm = __double2bfloat16(ci[v]);
            const double rr = cr[v] - (double)__bfloat162float(hr), ri = ci[v] - (double)__bfloat162float(hm);
            const __nv_bfloat16 mr = __double2bfloat16(rr), mi = __double2bfloat16(ri);
            const __nv_bfloat16 lr = __double2bfloat16(rr - (double)__bfloat162float(mr));
            const __nv_bfloat16 li = __double2bfloat16(ri - (double)__bfloat162float(mi));
            h[v] = bf16_pair(hr, hm);
            md[v] = bf16_pair(mr, mi);
            l[v] = bf16_pair(lr, li);
        }
        const uint32_t off = sw64_off(o, 8 * q4);
        *reinterpret_cast<uint4*>(cimg + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(cimg + kMsBBytes + off) = make_uint4(md[0], md[1], md[2], md[3]);
        *reinterpret_cast<uint4*>(cimg + 2 * kMsBBytes + off) = make_uint4(l[0], l[1], l[2], l[3]);
    } else if (F == kMsTf32) {
        uint32_t t[8];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            t[2 * v] = to_tf32((float)cr[v]);
            t[2 * v + 1] = to_tf32((float)ci[v]);
        }
        *reinterpret_cast<uint4*>(cimg + sw128_off(o, 8 * q4)) = make_uint4(t[0], t[1], t[2], t[3]);
        *reinterpret_cast<uint4*>(cimg + sw128_off(o, 8 * q4 + 4)) = make_uint4(t[4], t[5], t[6], t[7]);
    } else {
        uint32_t h[4], l[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float re = (float)cr[v], im = (float)ci[v];
            const __nv_bfloat16 hr = __float2bfloat16_rn(re), hm = __float2bfloat16_rn(im);
            const __nv_bfloat16 lr = __float2bfloat16_rn(re - __bfloat162float(hr));
            const __nv_bfloat16 li = __float2bfloat16_rn(im - __bfloat162float(hm));
            h[v] = bf16_pair(hr, hm);
            l[v] = bf16_pair(lr, li);
        }
        const uint32_t off = sw64_off(o, 8 * q4);
        *reinterpret_cast<uint4*>(cimg + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(cimg + kMsBBytes + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

// tile phases e^{i k_m r_n0}, r_n0 = (tile * 256 + 1) dr: the phase k r is
// reduced mod 2 pi in FP64 before the sine / cosine and the cast to FP32
// (tp64, when given, receives them in FP64, [tile][M_pad])
__device__ void ms_phase_entry(long long id, int M, int M_pad, int n_tiles, const double* __restrict__ kr,
                               const double* __restrict__ ki, double dr, int lossless, float2* __restrict__ q,
                               double2* __restrict__ tp64) {
    if (id >= (long long)n_tiles * M_pad) return;
    const int m = (int)(id % M_pad), tile = (int)(id / M_pad);
    if (m >= M) {
        q[id] = make_float2(0.f, 0.f);
        if (tp64) tp64[id] = make_double2(0.0, 0.0);
        return;
    }
    const double r = ((double)tile * kMsNT + 1.0) * dr;
    const double a = kr[m], b = lossless ? 0.0 : ki[m];
    const double th = a * r;
    const double turns = rint(th * (0.5 / kPi));
    const double red = fma(-turns, 2.0 * kPi, th);  // |red| <= pi (+ rounding)
    double sn, cs;
    sincos(red, &sn, &cs);
    const double amp = exp(-b * r);
    q[id] = make_float2((float)(amp * cs), (float)(amp * sn));
    if (tp64) tp64[id] = make_double2(amp * cs, amp * sn);
}

// A_jm = v_m(z_s) v_m(z_j) / sqrt(k_m) as complex FP32 for every receiver
// group and K-chunk, [group][chunk][mode m in chunk][receiver j in group];
// mode values at receiver j are row idx[j] of the full eigenvectors vfull
// [z][mode], vs the source values; zero for padding modes and receivers.
// a64, when given, receives A in FP64 as [receiver][M_pad] complex.
__device__ void ms_a_entry(long long id, int n_rcv, int M, int M_pad, int n_chunks, const double* __restrict__ kr,
                           const double* __restrict__ ki, const double* __restrict__ vs, const int* __restrict__ idx,
                           const double* __restrict__ vfull, int lossless, float2* __restrict__ ac,
                           double2* __restrict__ a64) {
    const int n_groups = (n_rcv + kMsRcv - 1) / kMsRcv;
    const long long per_chunk = (long long)kMsModes * kMsRcv;
    if (id >= (long long)n_groups * n_chunks * per_chunk) return;
    const int jl = (int)(id % kMsRcv);
    const int ml = (int)((id / kMsRcv) % kMsModes);
    const long long gc = id / per_chunk;  // group * n_chunks + chunk
    const int chunk = (int)(gc % n_chunks), g = (int)(gc / n_chunks);
    const int m = chunk * kMsModes + ml;
    const int j = g * kMsRcv + jl;
    float2 v = make_float2(0.f, 0.f);
    if (m < M && j < n_rcv) {
        const double a = kr[m], b = lossless ? 0.0 : ki[m];
        const auto sk = csqrt_principal(a, b);
        const double den = sk.real() * sk.real() + sk.imag() * sk.imag();
        const double c = vs[m] * vfull[(size_t)idx[j] * M + m];
        const double are = c * sk.real() / den, aim = -c * sk.imag() / den;
        v = make_float2((float)are, (float)aim);
        if (a64) a64[(size_t)j * M_pad + m] = make_double2(are, aim);
    }
    ac[id] = v;
}

// the three preparations in one launch: blocks [0, b_b) fill the B' images,
// [b_b, b_b + b_q) the tile phases, the rest A
// (the FP64 tables b64, tp64, a64 are written only for the guarded sum)
template <int F>
__global__ void k_ms_prepare(long long b_b, long long b_q, int n_rcv, int M, int M_pad, int n_tiles, int n_chunks,
                             const double* __restrict__ kr, const double* __restrict__ ki,
                             const double* __restrict__ vs, const int* __restrict__ idx,
                             const double* __restrict__ vfull, double dr, int lossless,
                             unsigned char* __restrict__ b_img, float2* __restrict__ q, float2* __restrict__ ac,
                             double2* __restrict__ b64, double2* __restrict__ tp64, double2* __restrict__ a64) {
    const long long b = blockIdx.x;
    if (b < b_b) {
        ms_b_entry<F>(b * blockDim.x + threadIdx.x, M, M_pad, n_chunks, kr, ki, dr, lossless, b_img, b64);
    } else if (b < b_b + b_q) {
        ms_phase_entry((b - b_b) * blockDim.x + threadIdx.x, M, M_pad, n_tiles, kr, ki, dr, lossless, q, tp64);
    } else {
        ms_a_entry((b - b_b - b_q) * blockDim.x + threadIdx.x, n_rcv, M, M_pad, n_chunks, kr, ki, vs, idx, vfull,
                   lossless, ac, a64);
    }
}

// ---------------------------------------------------------------------------
// the tensor-core kernel
// ---------------------------------------------------------------------------
// CTA that owns unit u when U units are split evenly over G CTAs (CTA b owns
// [floor(U b / G), floor(U (b + 1) / G)))
__host__ __device__ __forceinline__ int ms_cta_of(long long u, long long U, int G) {
    return (int)(((u + 1) * G - 1) / U);
}

struct MsArgs {
    const float2* ac;            // A: [groups][n_chunks][kMsModes][kMsRcv] complex FP32
    const float2* q;             // [n_tiles][M_pad]
    const unsigned char* b_img;  // B' images: [n_chunks][32 KB]
    int M_pad, n_chunks, n_tiles, n_ranges, groups;
    int acc_chunks;              // chunks per TMEM accumulation (the guarded sum's block)
    long long n_units;           // groups * n_tiles * n_chunks
    float* raw;                  // [n_parts][groups][n_tiles][256 columns][128 rows] per-CTA partial tiles
    float* s_part;               // guarded sum: [n_parts][groups][n_tiles][64 receivers][4] partial sums of |A'|
    unsigned* err;
};

// position of a CTA's current unit, advanced chunk by chunk without division;
// cib = the chunk's place in its accumulation block (blocks of acc_chunks
// chunks from the tile's first chunk)
struct UnitPos {
    int chunk, tile, group, cib;
    __device__ void init(long long u, int n_chunks, int n_tiles, int acc_chunks) {
        chunk = (int)(u % n_chunks);
        const long long gt = u / n_chunks;
        tile = (int)(gt % n_tiles);
        group = (int)(gt / n_tiles);
        cib = chunk % acc_chunks;
    }
    __device__ void next(int n_chunks, int n_tiles, int acc_chunks) {
        if (++cib == acc_chunks) cib = 0;
        if (++chunk == n_chunks) {
            chunk = 0;
            cib = 0;
            if (++tile == n_tiles) {
                tile = 0;
                ++group;
            }
        }
    }
};

template <int F, int TS, int GS>
__global__ void __launch_bounds__(kMsThreads, 1) k_ms_tc(MsArgs a) {
    using C = MsCfg<F, TS, GS>;
    constexpr int kTStages = C::kTStages, kGStages = C::kGStages;
    extern __shared__ unsigned char ms_dyn[];
    __shared__ __align__(8) uint64_t full_t[kMsMaxStages], empty_t[kMsMaxStages], full_g[kMsMaxStages],
        empty_g[kMsMaxStages];
    __shared__ __align__(8) uint64_t acc_full[kMsAcc], acc_empty[kMsAcc], drain;
    __shared__ uint32_t tmem_base_sh;
    unsigned char* sm = (unsigned char*)(((uintptr_t)ms_dyn + 1023) & ~(uintptr_t)1023);
    const uint32_t sm_addr = smem_u32(sm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this CTA's units [u0, u0 + nc), ordered (group, tile, chunk)
    const long long u0 = a.n_units * blockIdx.x / gridDim.x;
    const int nc = (int)(a.n_units * (blockIdx.x + 1) / gridDim.x - u0);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTStages; ++s) {
            mbar_init(&full_t[s], 1);
            mbar_init(&empty_t[s], 1);
        }
        for (int s = 0; s < kGStages; ++s) {
            mbar_init(&full_g[s], kMsGenWarps);
            mbar_init(&empty_g[s], 1);
        }
        for (int b = 0; b < kMsAcc; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kMsEpiWarps);
        }
        mbar_init(&drain, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(kMsAcc * kMsNT)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == kMsProducerWarp) {
        if (lane == 0 && nc > 0) {
            // producer: bulk TMA of the B' image, A and tile phases of chunk c
            // into TMA stage c % kTStages once the MMAs of chunk c - kTStages are done
            UnitPos pos;
            pos.init(u0, a.n_chunks, a.n_tiles, a.acc_chunks);
            int issued = 0, landed = 0;
            bool ok = true;
            for (int c = 0; c < nc; ++c, pos.next(a.n_chunks, a.n_tiles, a.acc_chunks)) {
                const int slot = c % kTStages;
                if (c >= kTStages) {
                    ok = mbar_wait_bounded(&empty_t[slot], (uint32_t)(((c / kTStages) - 1) & 1), a.err);
                    if (!ok) break;
                    landed = c - kTStages + 1;  // its copies were consumed, so they landed
                }
                unsigned char* dst = sm + slot * C::kTStageBytes;
                mbar_expect_tx(&full_t[slot], C::kTx);
                tma_load_1d(dst, a.b_img + (size_t)pos.chunk * C::kBChunk, C::kBChunk, &full_t[slot]);
                tma_load_1d(dst + C::kOffAC, a.ac + ((size_t)pos.group * a.n_chunks + pos.chunk) * kMsModes * kMsRcv,
                            kMsACBytes, &full_t[slot]);
                tma_load_1d(dst + C::kOffQ, a.q + (size_t)pos.tile * a.M_pad + pos.chunk * kMsModes, kMsQBytes,
                            &full_t[slot]);
                ++issued;
            }
            // copies still in flight after an early exit: wait for them
            for (int c = landed; c < issued; ++c)
                mbar_wait_drain(&full_t[c % kTStages], (uint32_t)((c / kTStages) & 1));
        }
    } else if (warp == 0) {
        if (lane == 0 && nc > 0) {
            // MMA issuer
            UnitPos pos;
            pos.init(u0, a.n_chunks, a.n_tiles, a.acc_chunks);
            bool ok = true;
            int sg = -1;  // segment (one group and tile) counter
            const uint64_t dsc0 = F == kMsTf32 ? smem_desc_sw128(sm_addr) : smem_desc(sm_addr);
            for (int c = 0; c < nc && ok; ++c, pos.next(a.n_chunks, a.n_tiles, a.acc_chunks)) {
                // one accumulation: this CTA's chunks of one tile inside one block
                const bool first = c == 0 || pos.cib == 0;
                const bool last = c == nc - 1 || pos.chunk == a.n_chunks - 1 || pos.cib == a.acc_chunks - 1;
                if (first) {
                    ++sg;
                    if (sg >= kMsAcc) {  // accumulator sg % 2 read out by the epilogue of segment sg - 2
                        ok = mbar_wait_bounded(&acc_empty[sg & 1], (uint32_t)(((sg >> 1) - 1) & 1), a.err);
                        if (!ok) break;
                        tc_fence_after();
                    }
                }
                const int stt = c % kTStages, sg_ = c % kGStages;
                ok = mbar_wait_bounded(&full_t[stt], (uint32_t)((c / kTStages) & 1), a.err) &&
                     mbar_wait_bounded(&full_g[sg_], (uint32_t)((c / kGStages) & 1), a.err);
                if (!ok) break;
                tc_fence_after();
                // descriptors: the start-address field counts 16-byte units;
                // A' from the generated ring, B' from the TMA stage
                const uint64_t st = dsc0 + (uint64_t)((C::kOffGRing + sg_ * C::kGStageBytes) >> 4);
                const uint64_t stb = dsc0 + (uint64_t)((stt * C::kTStageBytes) >> 4);
                const uint32_t d = tmem + (uint32_t)((sg & 1) * kMsNT);
                if (F == kMsTf32) {
                    // K = 8 tf32 (32 B) per MMA, four per chunk
#pragma unroll
                    for (int kk = 0; kk < kMsKC / 8; ++kk) {
                        const uint64_t ad = st + (uint64_t)(kk * 32 >> 4);
                        const uint64_t bd = stb + (uint64_t)(kk * 32 >> 4);
                        umma_tf32(d, ad, bd, (!first || kk > 0) ? 1u : 0u);
                    }
                } else if (F == kMsBf16x6) {
                    // six products; the three smallest first
#pragma unroll
                    for (int kk = 0; kk < kMsKC / 16; ++kk) {
                        const uint64_t ah = st + (uint64_t)(kk * 32 >> 4), am = ah + (uint64_t)(kMsABytes >> 4),
                                       al = am + (uint64_t)(kMsABytes >> 4);
                        const uint64_t bh = stb + (uint64_t)(kk * 32 >> 4), bm = bh + (uint64_t)(kMsBBytes >> 4),
                                       bl = bm + (uint64_t)(kMsBBytes >> 4);
                        umma_bf16(d, al, bh, (!first || kk > 0) ? 1u : 0u);
                        umma_bf16(d, am, bm, 1u);
                        umma_bf16(d, ah, bl, 1u);
                        umma_bf16(d, am, bh, 1u);
                        umma_bf16(d, ah, bm, 1u);
                        umma_bf16(d, ah, bh, 1u);
                    }
                } else {
#pragma unroll
                    for (int kk = 0; kk < kMsKC / 16; ++kk) {
                        const uint64_t ah = st + (uint64_t)(kk * 32 >> 4), al = ah + (uint64_t)(kMsABytes >> 4);
                        const uint64_t bh = stb + (uint64_t)(kk * 32 >> 4), bl = bh + (uint64_t)(kMsBBytes >> 4);
                        umma_bf16(d, ah, bh, (!first || kk > 0) ? 1u : 0u);
                        umma_bf16(d, ah, bl, 1u);
                        umma_bf16(d, al, bh, 1u);
                    }
                }
                umma_commit(&empty_t[stt]);
                umma_commit(&empty_g[sg_]);
                if (last) umma_commit(&acc_full[sg & 1]);
            }
            if (!ok) {
                // let the epilogue warps leave: a commit arrives once the
                // MMAs already issued are complete
                umma_commit(&acc_full[0]);
                umma_commit(&acc_full[1]);
            }
            // every MMA complete before the accumulators are released
            umma_commit(&drain);
            mbar_wait_drain(&drain, 0u);
        }
    } else if (warp <= kMsGenWarps) {
        // A' generators: thread -> (receiver j of the group, mode quad q4);
        // A'(tile) = A diag(e^{i k r_n0}) in the real block form
        // [[Re, -Im], [Im, Re]]: row j holds (Re, -Im) and row j + 64 (Im, Re)
        // of the 4 modes' products at k = 8 q4 .. 8 q4 + 7
        const int t = threadIdx.x - 32;
        const int j = t & (kMsRcv - 1), q4 = t >> 6;
        bool ok = true;
        float s_abs = 0.f;  // guarded sum: sum of |A'| over this thread's modes of the tile
        UnitPos pos;
        pos.init(u0, a.n_chunks, a.n_tiles, a.acc_chunks);
        for (int c = 0; c < nc && ok; ++c, pos.next(a.n_chunks, a.n_tiles, a.acc_chunks)) {
            const bool tile_first = c == 0 || pos.chunk == 0;
            const bool tile_last = c == nc - 1 || pos.chunk == a.n_chunks - 1;
            if (tile_first) s_abs = 0.f;
            const int stt = c % kTStages, sgs = c % kGStages;
            if (c >= kGStages) {  // A' stage free once the MMAs of chunk c - kGStages are done
                ok = mbar_wait_bounded(&empty_g[sgs], (uint32_t)(((c / kGStages) - 1) & 1), a.err);
                if (!ok) break;
            }
            ok = mbar_wait_bounded(&full_t[stt], (uint32_t)((c / kTStages) & 1), a.err);
            if (!ok) break;
            const unsigned char* stg = sm + stt * C::kTStageBytes;
            const float2* ac_s = reinterpret_cast<const float2*>(stg + C::kOffAC);
            const float2* q_s = reinterpret_cast<const float2*>(stg + C::kOffQ);
            float2 e[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) e[v] = cmulf(ac_s[(4 * q4 + v) * kMsRcv + j], q_s[4 * q4 + v]);
            const uint32_t gb = sm_addr + C::kOffGRing + sgs * C::kGStageBytes;
            if (F == kMsBf16x6) {
#pragma unroll
                for (int v = 0; v < 4; ++v) s_abs += sqrtf(fmaf(e[v].x, e[v].x, e[v].y * e[v].y));
                uint32_t hr[4], mr[4], lr[4], hm[4], mm[4], lm[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    split3(make_float2(e[v].x, -e[v].y), hr[v], mr[v], lr[v]);
                    split3(make_float2(e[v].y, e[v].x), hm[v], mm[v], lm[v]);
                }
                const uint32_t o0 = sw64_off(j, 8 * q4), o1 = sw64_off(j + kMsRcv, 8 * q4);
                sts128(gb + o0, hr[0], hr[1], hr[2], hr[3]);
                sts128(gb + kMsABytes + o0, mr[0], mr[1], mr[2], mr[3]);
                sts128(gb + 2 * kMsABytes + o0, lr[0], lr[1], lr[2], lr[3]);
                sts128(gb + o1, hm[0], hm[1], hm[2], hm[3]);
                sts128(gb + kMsABytes + o1, mm[0], mm[1], mm[2], mm[3]);
                sts128(gb + 2 * kMsABytes + o1, lm[0], lm[1], lm[2], lm[3]);
            } else if (F == kMsTf32) {
                const uint32_t r0 = gb + sw128_off(j, 8 * q4), r1 = gb + sw128_off(j + kMsRcv, 8 * q4);
                sts128(r0, to_tf32(e[0].x), to_tf32(-e[0].y), to_tf32(e[1].x), to_tf32(-e[1].y));
                sts128(gb + sw128_off(j, 8 * q4 + 4), to_tf32(e[2].x), to_tf32(-e[2].y), to_tf32(e[3].x),
                       to_tf32(-e[3].y));
                sts128(r1, to_tf32(e[0].y), to_tf32(e[0].x), to_tf32(e[1].y), to_tf32(e[1].x));
                sts128(gb + sw128_off(j + kMsRcv, 8 * q4 + 4), to_tf32(e[2].y), to_tf32(e[2].x), to_tf32(e[3].y),
                       to_tf32(e[3].x));
            } else {
                uint32_t hr[4], lr[4], hm[4], lm[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    split2(make_float2(e[v].x, -e[v].y), hr[v], lr[v]);
                    split2(make_float2(e[v].y, e[v].x), hm[v], lm[v]);
                }
                const uint32_t o0 = sw64_off(j, 8 * q4), o1 = sw64_off(j + kMsRcv, 8 * q4);
                sts128(gb + o0, hr[0], hr[1], hr[2], hr[3]);
                sts128(gb + kMsABytes + o0, lr[0], lr[1], lr[2], lr[3]);
                sts128(gb + o1, hm[0], hm[1], hm[2], hm[3]);
                sts128(gb + kMsABytes + o1, lm[0], lm[1], lm[2], lm[3]);
            }
            // every lane's writes visible to the tensor cores, then one
            // arrival per warp
            fence_proxy_async();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full_g[sgs])) : "memory");
            if (F == kMsBf16x6 && a.s_part && tile_last) {
                // the tile's sum of |A'| goes to slot (this CTA - first CTA of the tile)
                const long long gt = (long long)pos.group * a.n_tiles + pos.tile;
                const int part_slot = blockIdx.x - ms_cta_of(gt * a.n_chunks, a.n_units, gridDim.x);
                a.s_part[(((size_t)part_slot * a.groups + pos.group) * a.n_tiles + pos.tile) * (kMsRcv * 4) + j * 4 +
                         q4] = s_abs;
            }
        }
    } else if (warp >= kMsEpiWarp0) {
        // epilogue: thread -> accumulator row 32 (warp % 4) + lane (TMEM lane
        // quarter warp % 4), all kMsNT columns.  The partial sum of a tile
        // goes to slot (this CTA - first CTA of the tile), stored by the
        // tile's first accumulation and added to (FP32, round to nearest) by
        // the later ones; each thread reads back only the addresses it wrote
        // itself, kEpiAhead * kEpiCols columns ahead of the ones it adds.
        const int row = 32 * (warp & 3) + lane;
        bool ok = true;
        int sg = -1;
        bool fresh = true;  // no accumulation of this tile stored yet by this CTA
        UnitPos pos;
        pos.init(u0, a.n_chunks, a.n_tiles, a.acc_chunks);
        for (int c = 0; c < nc && ok; ++c, pos.next(a.n_chunks, a.n_tiles, a.acc_chunks)) {
            const bool tile_first = c == 0 || pos.chunk == 0;
            const bool tile_last = c == nc - 1 || pos.chunk == a.n_chunks - 1;
            if (tile_first) fresh = true;
            if (tile_first || pos.cib == 0) ++sg;
            if (!(tile_last || pos.cib == a.acc_chunks - 1)) continue;
            const long long gt = (long long)pos.group * a.n_tiles + pos.tile;
            const int part_slot = blockIdx.x - ms_cta_of(gt * a.n_chunks, a.n_units, gridDim.x);
            // partial tile stored column-major (the 128 rows of a column
            // contiguous), so each store instruction of the warp writes 128 B;
            // columns past n_ranges (last tile) land in the tile's own padding
            // and are never read
            float* tcol = a.raw + (((size_t)part_slot * a.groups + pos.group) * a.n_tiles + pos.tile) * kMsNT * kMsRows +
                          row;
            // old partial sums kEpiAhead column groups ahead of the adds (the
            // first ones loaded while the accumulator is still being filled)
            float o[kEpiAhead][kEpiCols];
            if (!fresh) {
#pragma unroll
                for (int d = 0; d < kEpiAhead; ++d)
#pragma unroll
                    for (int x = 0; x < kEpiCols; ++x) o[d][x] = tcol[(size_t)(d * kEpiCols + x) * kMsRows];
            }
            bool acc_ok = mbar_wait_bounded(&acc_full[sg & 1], (uint32_t)((sg >> 1) & 1), a.err);
            acc_ok = __all_sync(0xffffffffu, acc_ok);  // tcgen05.ld is warp-collective
            if (!acc_ok) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int cb = 0; cb < kMsNT / kEpiCols; ++cb) {
                uint32_t v[kEpiCols];
                const uint32_t taddr =
                    tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((sg & 1) * kMsNT + cb * kEpiCols);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float* tc = tcol + (size_t)(cb * kEpiCols) * kMsRows;
                float* slot = o[cb % kEpiAhead];
                if (fresh) {
#pragma unroll
                    for (int x = 0; x < kEpiCols; ++x) tc[(size_t)x * kMsRows] = __uint_as_float(v[x]);
                } else {
#pragma unroll
                    for (int x = 0; x < kEpiCols; ++x) tc[(size_t)x * kMsRows] = slot[x] + __uint_as_float(v[x]);
                    if (cb + kEpiAhead < kMsNT / kEpiCols) {
#pragma unroll
                        for (int x = 0; x < kEpiCols; ++x)
                            slot[x] = tc[(size_t)(kEpiAhead * kEpiCols + x) * kMsRows];
                    }
                }
            }
            fresh = false;
            tc_fence_before();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[sg & 1])) : "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMsAcc * kMsNT)
                     : "memory");
    }
}

// P = C(r_n) (D_re + i D_im) -> [n_rcv x n_ranges] FP64, adding the partial
// tiles of the CTAs that shared the tile (in FP64, slot order); C(r) =
// (cr + i ci) / sqrt(r).  Block = (group, tile, 32-column block): the columns
// are read contiguously (128 rows each), transposed through shared memory
// and written along the ranges.
//
// Guarded sum (s_part given): S_j = sum_m |A'_jm| over the tile (the sums the
// generators left in s_part) bounds sum_m |A_jm e^{i k_m r}| for every range
// of the tile, since |e^{i k r}| = e^{-Im k r} only falls with r.  A point
// whose |D| < tau S_j could carry more than the allowed TL error; it is
// appended to fix_list (receiver, range) for k_ms_fix.
constexpr int kMsFinCols = 32;
__global__ void __launch_bounds__(256) k_ms_finish(int n_rcv, int n_ranges, double dr, int groups, int n_tiles,
                                                   int n_chunks, long long n_units, int n_ctas, double cr, double ci,
                                                   const float* __restrict__ raw, double* __restrict__ re,
                                                   double* __restrict__ im, const float* __restrict__ s_part,
                                                   double tau, int* __restrict__ fix_count,
                                                   int2* __restrict__ fix_list) {
    __shared__ double sum[kMsFinCols][kMsRows + 1];
    __shared__ double sbound[kMsRcv];
    __shared__ int parts_sh;
    const int cb = blockIdx.x % (kMsNT / kMsFinCols);
    const int gt = blockIdx.x / (kMsNT / kMsFinCols);
    const int tile = gt % n_tiles, g = gt / n_tiles;
    if (threadIdx.x == 0) {
        const long long u_first = (long long)gt * n_chunks;
        parts_sh = ms_cta_of(u_first + n_chunks - 1, n_units, n_ctas) - ms_cta_of(u_first, n_units, n_ctas) + 1;
    }
    __syncthreads();
    const bool guard = s_part != nullptr;
    if (guard && threadIdx.x < kMsRcv) {
        double t = 0.0;
        for (int p = 0; p < parts_sh; ++p) {
            const float4 v = *reinterpret_cast<const float4*>(
                s_part + (((size_t)p * groups + g) * n_tiles + tile) * (kMsRcv * 4) + threadIdx.x * 4);
            t += (double)v.x + (double)v.y + (double)v.z + (double)v.w;
        }
        sbound[threadIdx.x] = t * tau;
    }
    const int c0 = cb * kMsFinCols;  // first column inside the tile
    const int row = threadIdx.x & (kMsRows - 1), col0 = threadIdx.x >> 7;
    // every slot read was written in full (256 columns, padding included)
    constexpr int kPer = kMsFinCols / 2;  // columns per thread
    double acc[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) acc[k] = 0.0;
    for (int p = 0; p < parts_sh; ++p) {
        const float* base = raw + ((((size_t)p * groups + g) * n_tiles + tile) * kMsNT + c0 + col0) * kMsRows + row;
        float v[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) v[k] = base[(size_t)(2 * k) * kMsRows];
#pragma unroll
        for (int k = 0; k < kPer; ++k) acc[k] += v[k];
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) sum[col0 + 2 * k][row] = acc[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int nl = threadIdx.x & (kMsFinCols - 1);
    const int n = tile * kMsNT + c0 + nl;
    const bool valid = n < n_ranges;
    const double sr = valid ? 1.0 / sqrt((n + 1) * dr) : 0.0;
    const double fr = cr * sr, fi = ci * sr;
    for (int jr = threadIdx.x >> 5; jr < kMsRcv; jr += 256 / kMsFinCols) {
        const int j = g * kMsRcv + jr;
        if (j >= n_rcv) break;  // the same for the whole warp
        const double dre = sum[nl][jr], dim = sum[nl][jr + kMsRcv];
        bool flag = false;
        if (valid) {
            const size_t o = (size_t)j * n_ranges + n;
            re[o] = fr * dre - fi * dim;
            im[o] = fr * dim + fi * dre;
            if (guard) {
                const double b = sbound[jr];
                flag = fma(dre, dre, dim * dim) < b * b;
            }
        }
        if (guard) {
            const unsigned bal = __ballot_sync(0xffffffffu, flag);
            if (bal) {
                int base = 0;
                if (lane == 0) base = atomicAdd(fix_count, __popc(bal));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (flag) fix_list[base + __popc(bal & ((1u << lane) - 1u))] = make_int2(j, n);
            }
        }
    }
}

// FP64 recomputation of the flagged points of the guarded sum, one warp per
// point: P = C(r) sum_m A_jm e^{i k_m r_n} with e^{i k r_n} = (tile phase)
// (offset phase), both FP64 tables of the preparation, the same
// factorisation as the tensor-core sum (r_n = r_n0 + o dr).
constexpr int kFixCtasPerSm = 4;
__global__ void __launch_bounds__(256) k_ms_fix(const int* __restrict__ fix_count, const int2* __restrict__ fix_list,
                                                int M, int M_pad, int n_ranges, double dr, double cr, double ci,
                                                const double2* __restrict__ a64, const double2* __restrict__ tp64,
                                                const double2* __restrict__ b64, double* __restrict__ re,
                                                double* __restrict__ im) {
    const int lane = threadIdx.x & 31;
    const int wpc = blockDim.x >> 5;
    const int cnt = *fix_count;
    // each CTA takes a contiguous block of the list: neighbouring entries
    // come from one finishing warp (one receiver, one tile), so their A and
    // tile-phase rows are shared through L1
    const int per_cta = (cnt + (int)gridDim.x - 1) / (int)gridDim.x;
    const int w0 = blockIdx.x * per_cta, w1 = min(w0 + per_cta, cnt);
    for (int w = w0 + (threadIdx.x >> 5); w < w1; w += wpc) {
        const int2 pt = fix_list[w];
        const int j = pt.x, n = pt.y;
        const int tile = n / kMsNT, o = n % kMsNT;
        const double2* ar = a64 + (size_t)j * M_pad;
        const double2* tr = tp64 + (size_t)tile * M_pad;
        const double2* br = b64 + (size_t)o * M_pad;
        double sre = 0.0, sim = 0.0;
        for (int m = lane; m < M; m += 32) {
            const double2 t = __ldg(tr + m), b = __ldg(br + m), av = __ldg(ar + m);
            const double er = fma(t.x, b.x, -t.y * b.y), ei = fma(t.x, b.y, t.y * b.x);
            sre = fma(av.x, er, fma(-av.y, ei, sre));
            sim = fma(av.x, ei, fma(av.y, er, sim));
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            sre += __shfl_xor_sync(0xffffffffu, sre, off);
            sim += __shfl_xor_sync(0xffffffffu, sim, off);
        }
        if (lane == 0) {
            const double sr = 1.0 / sqrt((n + 1) * dr);
            const double fr = cr * sr, fi = ci * sr;
            const size_t oo = (size_t)j * n_ranges + n;
            re[oo] = fr * sre - fi * sim;
            im[oo] = fr * sim + fi * sre;
        }
    }
}

// gather of the mode values at the receiver grid points: vz[j][m] = v[idx_j][m]
__global__ void k_ms_gather(int n_rcv, int M, const int* __restrict__ idx, const double* __restrict__ vfull,
                            double* __restrict__ vz) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)n_rcv * M) return;
    const int m = (int)(id % M), j = (int)(id / M);
    vz[id] = vfull[(size_t)idx[j] * M + m];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
MsPlan ms_plan(int n_rcv, int M, int n_ranges, int num_sms) {
    MsPlan p{};
    p.groups = (n_rcv + kMsRcv - 1) / kMsRcv;
    p.n_chunks = (M + kMsModes - 1) / kMsModes;
    p.M_pad = p.n_chunks * kMsModes;
    p.n_tiles = (n_ranges + kMsNT - 1) / kMsNT;
    p.n_units = (long long)p.groups * p.n_tiles * p.n_chunks;
    p.n_ctas = (int)std::min<long long>(num_sms, p.n_units);
    // CTAs sharing one (group, tile): each writes its own partial slot
    p.n_parts = 1;
    for (long long gt = 0; p.n_units > 0 && gt < (long long)p.groups * p.n_tiles; ++gt) {
        const long long uf = gt * p.n_chunks;
        const int parts = ms_cta_of(uf + p.n_chunks - 1, p.n_units, p.n_ctas) - ms_cta_of(uf, p.n_units, p.n_ctas) + 1;
        p.n_parts = std::max(p.n_parts, parts);
    }
    p.a_img_bytes = (size_t)p.groups * p.n_chunks * kMsACBytes;  // A, complex FP32
    p.q_bytes = (size_t)p.n_tiles * p.M_pad * sizeof(float2);
    p.tab_bytes = (size_t)p.n_chunks * MsCfg<kMsBf16x6>::kBChunk;  // B' images (room for three parts)
    p.raw_bytes = (size_t)p.n_parts * p.groups * p.n_tiles * kMsNT * kMsRows * sizeof(float);
    // guarded sum
    p.s_part_bytes = (size_t)p.n_parts * p.groups * p.n_tiles * kMsRcv * 4 * sizeof(float);
    p.b64_bytes = (size_t)kMsNT * p.M_pad * 16;
    p.tp64_bytes = (size_t)p.n_tiles * p.M_pad * 16;
    p.a64_bytes = (size_t)n_rcv * p.M_pad * 16;
    p.fix_list_bytes = (size_t)n_rcv * n_ranges * sizeof(int2);
    return p;
}

double ms_guard_eps(const MsPlan& p) {
    // the calibrated bound, plus one FP32 rounding (2^-24 of at most S) per
    // block addition beyond the calibration's: a CTA's share of a tile (at
    // most per_cta chunks) touches at most ceil(per_cta / B) + 1 blocks of B
    // chunks
    const long long per_cta = p.n_ctas > 0 ? (p.n_units + p.n_ctas - 1) / p.n_ctas : 0;
    const long long blocks = (p.n_chunks + kMsAccChunks - 1) / kMsAccChunks;
    const long long adds = std::max(0LL, std::min(blocks, (per_cta + kMsAccChunks - 1) / kMsAccChunks + 1) - 1);
    return kMsGuardEps + (double)std::max(0LL, adds - kMsGuardCalAdds) * std::ldexp(1.0, -24);
}

double ms_guard_tau(const MsPlan& p) {
    // |dTL| <= 0.05 dB needs |dP| <= d |P| with d = 1 - 10^(-0.05 / 20); with
    // |dP| <= eps S, a point with |P_tc| >= eps S (1 + 1 / d) satisfies it
    const double d = 1.0 - std::pow(10.0, -kMsGuardTlDb / 20.0);
    return ms_guard_eps(p) * (1.0 + 1.0 / d);
}

int launch_ms_gather(cudaStream_t st, int n_rcv, int M, const int* idx, const double* vfull, double* vz) {
    const long long n = (long long)n_rcv * M;
    if (n == 0) return 0;
    k_ms_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_rcv, M, idx, vfull, vz);
    return 1;
}

// a_img receives A (complex FP32), tab the B' images, q the tile phases
int launch_ms_prepare(cudaStream_t st, const MsPlan& p, int fmt, int n_rcv, int M, const double* kr,
                      const double* ki, const double* vs, const int* idx, const double* vfull, double dr, int lossless,
                      void* a_img, void* q, void* tab, void* b64, void* tp64, void* a64) {
    if (fmt != kMsBf16x3 && fmt != kMsTf32 && fmt != kMsBf16x6) return -1;
    const long long n_b = (long long)p.n_chunks * kMsNT * kMsBQuads;
    const long long n_q = (long long)p.n_tiles * p.M_pad;
    const long long n_a = (long long)p.groups * p.n_chunks * kMsModes * kMsRcv;
    const long long b_b = (n_b + 255) / 256, b_q = (n_q + 255) / 256, b_a = (n_a + 255) / 256;
    auto kern = fmt == kMsTf32 ? k_ms_prepare<kMsTf32>
                               : (fmt == kMsBf16x6 ? k_ms_prepare<kMsBf16x6> : k_ms_prepare<kMsBf16x3>);
    kern<<<(unsigned)(b_b + b_q + b_a), 256, 0, st>>>(b_b, b_q, n_rcv, M, p.M_pad, p.n_tiles, p.n_chunks, kr, ki, vs,
                                                     idx, vfull, dr, lossless, (unsigned char*)tab, (float2*)q,
                                                     (float2*)a_img, (double2*)b64, (double2*)tp64, (double2*)a64);
    return 1;
}

namespace {
// the schedules of each format: (TMA ring depth, generated-A' ring depth)
struct MsVariant {
    const void* fn;
    int smem, ts, gs;
};
template <int F, int TS, int GS>
MsVariant ms_variant() {
    return MsVariant{(const void*)k_ms_tc<F, TS, GS>, MsCfg<F, TS, GS>::kSmem, TS, GS};
}
constexpr int kMsVariants = 4;
const MsVariant& ms_variant_of(int fmt, int v) {
    static const MsVariant x3[kMsVariants] = {ms_variant<kMsBf16x3, 4, 3>(), ms_variant<kMsBf16x3, 3, 3>(),
                                              ms_variant<kMsBf16x3, 4, 2>(), ms_variant<kMsBf16x3, 2, 3>()};
    static const MsVariant tf[kMsVariants] = {ms_variant<kMsTf32, 4, 3>(), ms_variant<kMsTf32, 3, 3>(),
                                              ms_variant<kMsTf32, 4, 2>(), ms_variant<kMsTf32, 2, 3>()};
    static const MsVariant x6[kMsVariants] = {ms_variant<kMsBf16x6, 3, 2>(), ms_variant<kMsBf16x6, 2, 3>(),
                                              ms_variant<kMsBf16x6, 2, 2>(), ms_variant<kMsBf16x6, 3, 1>()};
    return fmt == kMsTf32 ? tf[v] : (fmt == kMsBf16x6 ? x6[v] : x3[v]);
}
}  // namespace

int ms_tc_variants() { return kMsVariants; }

int ms_tile_ranges() { return kMsNT; }

void ms_tc_variant_shape(int fmt, int variant, int* t_stages, int* g_stages) {
    const MsVariant& v = ms_variant_of(fmt, variant < 0 || variant >= kMsVariants ? 0 : variant);
    *t_stages = v.ts;
    *g_stages = v.gs;
}

int launch_ms_tc(cudaStream_t st, const MsPlan& p, int fmt, int n_ranges, const void* a_img, const void* q,
                 const void* tab, float* raw, float* s_part, unsigned* err, int variant) {
    if (p.n_units <= 0) return 0;
    if (fmt != kMsBf16x3 && fmt != kMsTf32 && fmt != kMsBf16x6) return -1;
    if (variant < 0 || variant >= kMsVariants) return -1;
    const MsVariant& var = ms_variant_of(fmt, variant);
    static bool attr_set[3][kMsVariants][64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    if (!attr_set[fmt][variant][dev]) {
        if (cudaFuncSetAttribute(var.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, var.smem) != cudaSuccess)
            return -1;
        attr_set[fmt][variant][dev] = true;  // setting it twice from two threads is harmless
    }
    MsArgs a;
    a.ac = (const float2*)a_img;
    a.q = (const float2*)q;
    a.b_img = (const unsigned char*)tab;
    a.M_pad = p.M_pad;
    a.n_chunks = p.n_chunks;
    a.n_tiles = p.n_tiles;
    a.n_ranges = n_ranges;
    a.groups = p.groups;
    a.n_units = p.n_units;
    a.acc_chunks = fmt == kMsBf16x6 ? std::min(kMsAccChunks, p.n_chunks) : p.n_chunks;
    a.raw = raw;
    a.s_part = fmt == kMsBf16x6 ? s_part : nullptr;
    a.err = err;
    void* args[] = {&a};
    if (cudaLaunchKernel(var.fn, dim3(p.n_ctas), dim3(kMsThreads), args, (size_t)var.smem, st) != cudaSuccess)
        return -1;
    return 1;
}

namespace {
// 1000 * 4 pi i e^{-i pi/4} / sqrt(8 pi) = c0 (cos pi/4 + i sin pi/4)
void ms_scale(double& cr, double& ci) {
    const double c0 = 1000.0 * 4 * kPi / std::sqrt(8.0 * kPi);
    cr = c0 * std::sin(kPi * 0.25);
    ci = c0 * std::cos(kPi * 0.25);
}
}  // namespace

int launch_ms_finish(cudaStream_t st, const MsPlan& p, int n_rcv, int n_ranges, double dr, const float* raw,
                     double* re, double* im, const float* s_part, int* fix_count, void* fix_list) {
    double cr, ci;
    ms_scale(cr, ci);
    const unsigned blocks = (unsigned)(p.groups * p.n_tiles * (kMsNT / kMsFinCols));
    k_ms_finish<<<blocks, 256, 0, st>>>(n_rcv, n_ranges, dr, p.groups, p.n_tiles, p.n_chunks, p.n_units, p.n_ctas, cr,
                                        ci, raw, re, im, s_part, s_part ? ms_guard_tau(p) : 0.0, fix_count,
                                        (int2*)fix_list);
    return 1;
}

int launch_ms_fix(cudaStream_t st, int num_sms, int M, int M_pad, int n_ranges, double dr, const int* fix_count,
                  const void* fix_list, const void* a64, const void* tp64, const void* b64, double* re, double* im) {
    double cr, ci;
    ms_scale(cr, ci);
    k_ms_fix<<<kFixCtasPerSm * num_sms, 256, 0, st>>>(fix_count, (const int2*)fix_list, M, M_pad, n_ranges, dr, cr, ci,
                                          (const double2*)a64, (const double2*)tp64, (const double2*)b64, re, im);
    return 1;
}

}  // namespace ncpa
