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
// Each operand is split into bf16 hi + lo parts and D accumulates
//   A_hi B_hi + A_hi B_lo + A_lo B_hi   in FP32 (3-term split-BF16, ~2^-16).
//
// One CTA = one tile of 128 ranges x one K-range of modes (split-K when the
// tiles alone cannot fill the SMs).  Warp 0: TMEM allocation, bulk-TMA of
// the prepared A' chunks, tcgen05.mma issue.  Warps 1-4: generate B' in
// shared memory from FP64-reduced tile phases (e^{i k r_n0}, computed in
// FP64 with the phase reduced mod 2 pi) times short FP32 recurrences
// e^{i k 8 dr}, then read the accumulator out of TMEM.
//
// Shared-memory operand layout (no swizzle, K-major core matrices): element
// (row, k) of a 128-row x 64-k bf16 tile sits at byte
//   ((row / 8) * 8 + k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// i.e. leading-byte offset 128 (next 8 k) and stride-byte offset 1024 (next 8
// rows); one MMA (K = 16) starts 256 bytes further per K-step.
#include <cuda_bf16.h>

#include "device_common.cuh"

namespace ncpa {

namespace {

constexpr int kMsRows = 128;        // UMMA M (Re / Im rows of 64 receivers)
constexpr int kMsRcv = 64;          // receivers per group
constexpr int kMsNT = 128;          // ranges per tile (UMMA N)
constexpr int kMsModes = 32;        // modes per K-chunk
constexpr int kMsKC = 2 * kMsModes; // K per chunk
constexpr int kMsStages = 3;
constexpr int kMsOpBytes = kMsRows * kMsKC * 2;  // one operand part: 16 KB
constexpr int kMsStageBytes = 4 * kMsOpBytes;    // A hi, A lo, B hi, B lo
constexpr int kMsSmem = kMsStages * kMsStageBytes + 1024;
constexpr int kMsThreads = 160;
constexpr int kMsTabW = 10;         // per-mode table: 8 x e^{ik i dr}, e^{ik 64dr}, e^{ik 8dr}
static_assert(kMsNT == kMsRows, "square operand tiles share one layout");

__device__ __forceinline__ uint32_t core_off(int row, int k) {
    return (uint32_t)((((row >> 3) * (kMsKC / 8)) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (tcgen05 format): start >> 4 in [0,14),
// leading-byte offset >> 4 in [16,30), stride-byte offset >> 4 in [32,46),
// descriptor version 1 in [46,48), no swizzle (layout type 0 in [61,64))
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
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

__device__ __forceinline__ void sts128(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
                 : "memory");
}

}  // namespace

// ---------------------------------------------------------------------------
// preparation
// ---------------------------------------------------------------------------
// per-mode FP32 factors from FP64: e^{i k i dr} (i < 8), e^{i k 64 dr},
// e^{i k 8 dr}; zero for the padding modes m >= M
__global__ void k_ms_tables(int M, int M_pad, const double* __restrict__ kr, const double* __restrict__ ki,
                            double dr, int lossless, float2* __restrict__ tab) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M_pad) return;
    float2* t = tab + (size_t)m * kMsTabW;
    if (m >= M) {
        for (int i = 0; i < kMsTabW; ++i) t[i] = make_float2(0.f, 0.f);
        return;
    }
    const double a = kr[m], b = lossless ? 0.0 : ki[m];
    const double steps[kMsTabW] = {0, 1, 2, 3, 4, 5, 6, 7, 64, 8};
    for (int i = 0; i < kMsTabW; ++i) {
        const double x = steps[i] * dr;
        double sn, cs;
        sincos(a * x, &sn, &cs);
        const double amp = exp(-b * x);
        t[i] = make_float2((float)(amp * cs), (float)(amp * sn));
    }
}

// tile phases e^{i k_m r_n0}, r_n0 = (tile * 128 + 1) dr: the phase k r is
// reduced mod 2 pi in FP64 before the sine / cosine and the cast to FP32
__global__ void k_ms_phase(int M, int M_pad, int n_tiles, const double* __restrict__ kr,
                           const double* __restrict__ ki, double dr, int lossless, float2* __restrict__ q) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)n_tiles * M_pad) return;
    const int m = (int)(id % M_pad), tile = (int)(id / M_pad);
    if (m >= M) {
        q[id] = make_float2(0.f, 0.f);
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
}

// A' chunk images (hi, lo) for every receiver group and K-chunk, in the
// shared-memory layout above; vz is [n_rcv x M] (mode values at the
// receiver grid points), vs the source values
__global__ void k_ms_a(int n_rcv, int M, int n_chunks, const double* __restrict__ kr, const double* __restrict__ ki,
                       const double* __restrict__ vs, const double* __restrict__ vz, int lossless,
                       __nv_bfloat16* __restrict__ img) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n_groups = (n_rcv + kMsRcv - 1) / kMsRcv;
    const long long per_chunk = (long long)kMsRows * kMsKC;
    if (id >= (long long)n_groups * n_chunks * per_chunk) return;
    const int row = (int)(id % kMsRows);
    const int kl = (int)((id / kMsRows) % kMsKC);
    const long long gc = id / per_chunk;  // group * n_chunks + chunk
    const int chunk = (int)(gc % n_chunks), g = (int)(gc / n_chunks);
    const int m = chunk * kMsModes + (kl >> 1);
    const int j = g * kMsRcv + (row & (kMsRcv - 1));
    float x = 0.f;
    if (m < M && j < n_rcv) {
        const double a = kr[m], b = lossless ? 0.0 : ki[m];
        const auto sk = csqrt_principal(a, b);
        const double den = sk.real() * sk.real() + sk.imag() * sk.imag();
        const double c = vs[m] * vz[(size_t)j * M + m];
        const double are = c * sk.real() / den, aim = -c * sk.imag() / den;
        const bool im_row = row >= kMsRcv, im_col = (kl & 1) != 0;
        x = (float)(!im_row ? (im_col ? -aim : are) : (im_col ? are : aim));
    }
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
    const size_t base = (size_t)gc * 2 * (kMsOpBytes / 2);  // elements
    const size_t off = core_off(row, kl) / 2;
    img[base + off] = hi;
    img[base + kMsOpBytes / 2 + off] = lo;
}

// ---------------------------------------------------------------------------
// the tensor-core kernel
// ---------------------------------------------------------------------------
struct MsArgs {
    const unsigned char* a_img;  // [groups][n_chunks][hi, lo][16 KB]
    const float2* q;             // [n_tiles][M_pad]
    const float2* tab;           // [M_pad][10]
    int M_pad, n_chunks, chunks_per_split, n_splits, n_tiles, n_ranges;
    float* raw;                  // [groups][128][n_ranges] FP32 sums (zeroed when n_splits > 1)
    unsigned* err;
};

__global__ void __launch_bounds__(kMsThreads, 1) k_ms_tc(MsArgs a) {
    extern __shared__ unsigned char ms_dyn[];
    __shared__ __align__(8) uint64_t full_a[kMsStages], full_b[kMsStages], empty[kMsStages], acc_full;
    __shared__ uint32_t tmem_base_sh;
    unsigned char* sm = (unsigned char*)(((uintptr_t)ms_dyn + 1023) & ~(uintptr_t)1023);
    const uint32_t sm_addr = smem_u32(sm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x / a.n_splits, split = blockIdx.x % a.n_splits;
    const int group = blockIdx.y;
    const int c_begin = split * a.chunks_per_split;
    const int nc = min(a.chunks_per_split, a.n_chunks - c_begin);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kMsStages; ++s) {
            mbar_init(&full_a[s], 1);
            mbar_init(&full_b[s], 128);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&acc_full, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(kMsNT)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        if (lane == 0 && nc > 0) {
            // producer of A' (bulk TMA) and MMA issuer
            const unsigned char* src = a.a_img + ((size_t)group * a.n_chunks + c_begin) * 2 * kMsOpBytes;
            int issued = 0;
            for (; issued < min(kMsStages, nc); ++issued) {
                mbar_expect_tx(&full_a[issued], 2 * kMsOpBytes);
                tma_load_1d(sm + issued * kMsStageBytes, src + (size_t)issued * 2 * kMsOpBytes, 2 * kMsOpBytes,
                            &full_a[issued]);
            }
            bool ok = true;
            int waited_a = 0;  // chunks whose A' copy is known to have landed
            for (int c = 0; c < nc && ok; ++c) {
                const int s = c % kMsStages;
                const uint32_t ph = (uint32_t)((c / kMsStages) & 1);
                ok = mbar_wait_bounded(&full_a[s], ph, a.err);
                if (!ok) break;
                waited_a = c + 1;
                ok = mbar_wait_bounded(&full_b[s], ph, a.err);
                if (!ok) break;
                tc_fence_after();
                const uint32_t st = sm_addr + s * kMsStageBytes;
#pragma unroll
                for (int kk = 0; kk < kMsKC / 16; ++kk) {
                    const uint32_t ah = st + kk * 256, al = ah + kMsOpBytes;
                    const uint32_t bh = st + 2 * kMsOpBytes + kk * 256, bl = bh + kMsOpBytes;
                    umma_bf16(tmem, smem_desc(ah), smem_desc(bh), (c > 0 || kk > 0) ? 1u : 0u);
                    umma_bf16(tmem, smem_desc(ah), smem_desc(bl), 1u);
                    umma_bf16(tmem, smem_desc(al), smem_desc(bh), 1u);
                }
                umma_commit(&empty[s]);
                // refill the slot of chunk c - 1 once its MMAs are done
                if (c >= 1 && issued < nc) {
                    const int sp = (c - 1) % kMsStages;
                    ok = mbar_wait_bounded(&empty[sp], (uint32_t)(((c - 1) / kMsStages) & 1), a.err);
                    if (!ok) break;
                    mbar_expect_tx(&full_a[sp], 2 * kMsOpBytes);
                    tma_load_1d(sm + sp * kMsStageBytes, src + (size_t)issued * 2 * kMsOpBytes, 2 * kMsOpBytes,
                                &full_a[sp]);
                    ++issued;
                }
            }
            umma_commit(&acc_full);
            // copies still in flight after an early exit: wait for them
            for (int c = waited_a; c < issued; ++c)
                mbar_wait_drain(&full_a[c % kMsStages], (uint32_t)((c / kMsStages) & 1));
        }
    } else {
        // B' generators: thread -> (i = range in its 8-group, q = mode quad,
        // half = which 64 ranges)
        const int t = threadIdx.x - 32;
        const int i = t & 7, q = (t >> 3) & 7, half = t >> 6;
        const float2* qrow = a.q + (size_t)tile * a.M_pad;
        bool ok = true;
        for (int c = 0; c < nc && ok; ++c) {
            const int s = c % kMsStages;
            if (c >= kMsStages) {
                ok = mbar_wait_bounded(&empty[s], (uint32_t)(((c / kMsStages) - 1) & 1), a.err);
                if (!ok) break;
            }
            const int m0 = (c_begin + c) * kMsModes + 4 * q;
            float2 e[4], w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float2* tb = a.tab + (size_t)(m0 + u) * kMsTabW;
                float2 v = cmulf(qrow[m0 + u], tb[i]);
                if (half) v = cmulf(v, tb[8]);
                e[u] = v;
                w[u] = tb[9];
            }
            const uint32_t bh = sm_addr + s * kMsStageBytes + 2 * kMsOpBytes;
#pragma unroll
            for (int st8 = 0; st8 < 8; ++st8) {
                const int grp = half * 8 + st8;  // 8-range group within the tile
                const uint32_t off = (uint32_t)((grp * (kMsKC / 8) + q) * 128 + i * 16);
                uint32_t h[4], l[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) split2(e[u], h[u], l[u]);
                sts128(bh + off, h[0], h[1], h[2], h[3]);
                sts128(bh + kMsOpBytes + off, l[0], l[1], l[2], l[3]);
#pragma unroll
                for (int u = 0; u < 4; ++u) e[u] = cmulf(e[u], w[u]);
            }
            fence_proxy_async();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full_b[s])) : "memory");
        }
        // epilogue: TMEM lanes 32 (warp % 4) .. +31 = rows of D
        bool acc_ok = nc > 0 && mbar_wait_bounded(&acc_full, 0u, a.err);
        acc_ok = __all_sync(0xffffffffu, acc_ok);  // tcgen05.ld is warp-collective
        if (acc_ok) {
            tc_fence_after();
            const int row = 32 * (warp & 3) + lane;
            const int n0 = tile * kMsNT;
            float* out = a.raw + ((size_t)group * kMsRows + row) * a.n_ranges;
#pragma unroll 1
            for (int cb = 0; cb < kMsNT / 32; ++cb) {
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(cb * 32);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                    "%30, %31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int u = 0; u < 32; ++u) {
                    const int n = n0 + cb * 32 + u;
                    if (n < a.n_ranges) {
                        const float x = __uint_as_float(v[u]);
                        if (a.n_splits > 1) atomicAdd(out + n, x);
                        else out[n] = x;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMsNT) : "memory");
    }
}

// P = C(r_n) (D_re + i D_im) -> [n_rcv x n_ranges] FP64
__global__ void k_ms_finish(int n_rcv, int n_ranges, double dr, const float* __restrict__ raw,
                            double* __restrict__ re, double* __restrict__ im) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)n_rcv * n_ranges) return;
    const int n = (int)(id % n_ranges), j = (int)(id / n_ranges);
    const int g = j / kMsRcv, jr = j % kMsRcv;
    const float* base = raw + (size_t)g * kMsRows * n_ranges;
    const double dre = base[(size_t)jr * n_ranges + n], dim = base[(size_t)(jr + kMsRcv) * n_ranges + n];
    const double r = (n + 1) * dr;
    const double c0 = 1000.0 * 4 * kPi / sqrt(8.0 * kPi) / sqrt(r);
    const double fr = c0 * sin(kPi * 0.25), fi = c0 * cos(kPi * 0.25);
    re[id] = fr * dre - fi * dim;
    im[id] = fr * dim + fi * dre;
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
    // split K until the CTAs cover the SMs (about two per SM), keeping at
    // least four chunks per split so the pipeline fills
    const int units = p.n_tiles * p.groups;
    int splits = 1;
    while (units * splits < 2 * num_sms && p.n_chunks / (splits * 2) >= 4) splits *= 2;
    p.chunks_per_split = (p.n_chunks + splits - 1) / splits;
    p.n_splits = (p.n_chunks + p.chunks_per_split - 1) / p.chunks_per_split;
    p.a_img_bytes = (size_t)p.groups * p.n_chunks * 2 * kMsOpBytes;
    p.q_bytes = (size_t)p.n_tiles * p.M_pad * sizeof(float2);
    p.tab_bytes = (size_t)p.M_pad * kMsTabW * sizeof(float2);
    p.raw_bytes = (size_t)p.groups * kMsRows * n_ranges * sizeof(float);
    return p;
}

int launch_ms_gather(cudaStream_t st, int n_rcv, int M, const int* idx, const double* vfull, double* vz) {
    const long long n = (long long)n_rcv * M;
    if (n == 0) return 0;
    k_ms_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_rcv, M, idx, vfull, vz);
    return 1;
}

int launch_ms_prepare(cudaStream_t st, const MsPlan& p, int n_rcv, int M, const double* kr, const double* ki,
                      const double* vs, const double* vz, double dr, int lossless, void* a_img, void* q, void* tab) {
    k_ms_tables<<<(p.M_pad + 127) / 128, 128, 0, st>>>(M, p.M_pad, kr, ki, dr, lossless, (float2*)tab);
    const long long nq = (long long)p.n_tiles * p.M_pad;
    k_ms_phase<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(M, p.M_pad, p.n_tiles, kr, ki, dr, lossless,
                                                              (float2*)q);
    const long long na = (long long)p.groups * p.n_chunks * kMsRows * kMsKC;
    k_ms_a<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(n_rcv, M, p.n_chunks, kr, ki, vs, vz, lossless,
                                                          (__nv_bfloat16*)a_img);
    return 3;
}

int launch_ms_tc(cudaStream_t st, const MsPlan& p, int n_ranges, const void* a_img, const void* q, const void* tab,
                 float* raw, unsigned* err) {
    if (cudaFuncSetAttribute(k_ms_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kMsSmem) != cudaSuccess)
        return -1;
    if (p.n_splits > 1) cudaMemsetAsync(raw, 0, p.raw_bytes, st);
    MsArgs a;
    a.a_img = (const unsigned char*)a_img;
    a.q = (const float2*)q;
    a.tab = (const float2*)tab;
    a.M_pad = p.M_pad;
    a.n_chunks = p.n_chunks;
    a.chunks_per_split = p.chunks_per_split;
    a.n_splits = p.n_splits;
    a.n_tiles = p.n_tiles;
    a.n_ranges = n_ranges;
    a.raw = raw;
    a.err = err;
    dim3 grid(p.n_tiles * p.n_splits, p.groups);
    k_ms_tc<<<grid, kMsThreads, kMsSmem, st>>>(a);
    return 1;
}

int launch_ms_finish(cudaStream_t st, int n_rcv, int n_ranges, double dr, const float* raw, double* re, double* im) {
    const long long n = (long long)n_rcv * n_ranges;
    k_ms_finish<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_rcv, n_ranges, dr, raw, re, im);
    return 1;
}

}  // namespace ncpa
