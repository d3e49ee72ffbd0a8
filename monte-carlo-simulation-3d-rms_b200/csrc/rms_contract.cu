// rms_contract.cu -- the multi-waveform phase contraction.
//
// For walker trajectories sampled on time bins, pos[w][b][axis] (um; the
// walk's bin means, RMS_MODE_WAVEFORM with a trajectory output) and gradient
// waveforms wave[j][b][axis] (phase per um of a bin's position), the phase
// of walker w under waveform j is the contraction over K = 3 nbins
//
//     phi[w][j] = sum_k pos[w][k] wave[j][k],
//
// and the signal is (sum_w cos phi, sum_w sin phi) per waveform.  Walkers x
// waveforms x K is GEMM-shaped, so it runs on the tensor cores; phi never
// reaches memory: the epilogue turns each accumulator tile into cosine and
// sine sums.  There is no counterpart in the reference, whose only gradient
// form is the PGSE pair (hpc_code/lib/main_PGSE.cu:336-346), accumulated per
// step per gradient.
//
// Three methods:
//  - FP32 on the CUDA cores (contract_f32_kernel): register-tiled, 128
//    waveforms x 128 walkers per block;
//  - positions already split into BF16 pairs by the walk
//    (contract_presplit_kernel): the pipeline below with one TMA warp in
//    place of the converters (two tensor maps, hi and lo, 128-byte swizzle:
//    the tiles land in the MMA's operand layout as they are);
//  - BF16 hi/lo on the tensor cores (contract_tc_kernel): x = x_hi + x_lo with
//    both parts BF16, phi = A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in
//    FP32 in tensor memory (the dropped A_lo B_lo term is below 2^-16 of each
//    product).  tcgen05.mma kind::f16, M = 128 waveforms, N = 256 walkers,
//    K = 16 per instruction, one CTA per SM.  A work unit is 256 walkers x
//    two waveform tiles (256 waveforms): each converted position chunk feeds
//    the MMAs of both tiles, which halves the position loads per MMA.
//      warps 0-7  FP32 positions straight from global memory (the next half
//                 chunk's loads in flight while this one converts) -> BF16
//                 hi/lo in the MMA's K-major 128-byte-swizzled layout, 2 stages
//      warp 12    bulk copies of the pre-split waveform tiles, 3 stages
//      warp 13    TMEM allocation, MMA issue (one thread), commits
//      warps 8-11 epilogue: tcgen05.ld of 32-column slices, range reduction,
//                 sine/cosine, per-row sums; FP64 atomics into the totals
//    The two tiles' accumulators fill the 512 TMEM columns; each has its own
//    full/empty barriers, so the next unit's MMAs into the first tile start
//    while the epilogue still reads the second.  Work units (walker tile,
//    waveform tile pair) are ordered pair fastest, so the CTAs reading one
//    walker tile run at the same time and share it in L2.  Every wait is bounded
//    (4 s of global time); a wait that runs out sets an error bit, the CTA
//    drains its copies and MMAs, frees its tensor memory and returns.
#include <cuda.h>   // CUtensorMap and the encoder's signature (fetched through cudaGetDriverEntryPoint)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/rms.h"
#include "rms_internal.h"

namespace rms {
namespace {

// ----------------------------------------------------------------------------
// shared pieces

// sin and cos of a phase on the FMA pipe only (the epilogue evaluates one
// pair per walker and waveform, ~1e10 pairs, which would saturate the
// special-function unit).  Quadrant q = round(phi 2/pi) by the 1.5 2^23
// rounding trick (|phi| < 2^21), r = phi - q pi/2 with pi/2 split into a float
// and its remainder (Cody-Waite), |r| <= pi/4; then the Taylor series of sin
// to r^9 and of cos to r^10 (truncation below 3e-8 there), swapped and negated
// by q mod 4.  Absolute error ~1e-7 for |phi| up to ~1e3.
__device__ __forceinline__ void sincos_reduced(float phi, float* s, float* c) {
    const float t = fmaf(phi, 0.636619772367581343f, 12582912.0f);
    const float q = t - 12582912.0f;
    const int quad = __float_as_int(t) & 3;
    float r = fmaf(-q, 1.57079637050628662f, phi);
    r = fmaf(q, 4.37113900018624284e-08f, r);
    const float z = r * r;
    float ps = fmaf(z, 2.75573192239858907e-06f, -1.98412698412698413e-04f);
    ps = fmaf(z, ps, 8.33333333333333333e-03f);
    ps = fmaf(z, ps, -1.66666666666666667e-01f);
    const float sn = fmaf(r * z, ps, r);
    float pc = fmaf(z, -2.75573192239858907e-07f, 2.48015873015873016e-05f);
    pc = fmaf(z, pc, -1.38888888888888889e-03f);
    pc = fmaf(z, pc, 4.16666666666666667e-02f);
    pc = fmaf(z, pc, -0.5f);
    const float cs = fmaf(z, pc, 1.0f);
    // (sin, cos)(r + q pi/2): q = 0 (s, c), 1 (c, -s), 2 (-s, -c), 3 (-c, s)
    const float a = (quad & 1) ? cs : sn;
    const float b = (quad & 1) ? sn : cs;
    *s = (quad & 2) ? -a : a;
    *c = ((quad + 1) & 2) ? -b : b;
}

// ----------------------------------------------------------------------------
// FP32 CUDA-core method

constexpr int kF32Tile = 128;   // waveforms and walkers per block
constexpr int kF32Kc = 16;

__global__ void __launch_bounds__(256) contract_f32_kernel(const float* __restrict__ pos, int64_t nwalk, int K,
                                                           const float* __restrict__ wave, int nwave,
                                                           int n_mtiles, double* __restrict__ out) {
    __shared__ float As[kF32Kc][kF32Tile];   // waveforms, [k][m]
    __shared__ float Bs[kF32Kc][kF32Tile];   // walkers, [k][n]
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int mt = (int)(blockIdx.x % n_mtiles);
    const int64_t wt = blockIdx.x / n_mtiles;
    const int m0 = mt * kF32Tile;
    const int64_t n0 = wt * kF32Tile;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;

    for (int k0 = 0; k0 < K; k0 += kF32Kc) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int e = tid + 256 * r;         // 0 .. 2047
            const int k = e & 15, row = e >> 4;  // 16 consecutive threads read one row's 16 k
            const int m = m0 + row;
            const int64_t n = n0 + row;
            As[k][row] = (m < nwave && k0 + k < K) ? __ldg(wave + (size_t)m * K + k0 + k) : 0.0f;
            Bs[k][row] = (n < nwalk && k0 + k < K) ? __ldg(pos + (size_t)n * K + k0 + k) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kF32Kc; ++k) {
            float a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    // epilogue: per waveform row, cosine and sine sums over this block's walkers
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float cs = 0.0f, sn = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float s, c;
            sincos_reduced(acc[i][j], &s, &c);
            const float m = (n0 + tx + 16 * j < nwalk) ? 1.0f : 0.0f;
            cs = fmaf(m, c, cs);
            sn = fmaf(m, s, sn);
        }
        // the 16 threads of a row (tx = 0..15) are 16 consecutive lanes
#pragma unroll
        for (int o = 8; o >= 1; o >>= 1) {
            cs += __shfl_xor_sync(0xffffffffu, cs, o);
            sn += __shfl_xor_sync(0xffffffffu, sn, o);
        }
        const int m = m0 + ty + 16 * i;
        if (tx == 0 && m < nwave) {
            atomicAdd(out + 2 * m, (double)cs);
            atomicAdd(out + 2 * m + 1, (double)sn);
        }
    }
}

// ----------------------------------------------------------------------------
// tensor-core method

constexpr int kKc = 64;                         // k per pipeline chunk: one 128-byte BF16 row
constexpr int kTileN = 256;                     // walkers per tile (MMA N)
constexpr int kTileM = 128;                     // waveforms per tile (MMA M)
constexpr int kBStages = 2;                     // converted position chunks
constexpr int kGStages = 3;                     // waveform chunks of one tile (a copy is issued once an MMA frees one)
constexpr uint32_t kXbBytes = kTileN * kKc * 2;         // one BF16 part: 32768
constexpr uint32_t kGBytes = kTileM * kKc * 2;          // one BF16 part: 16384
constexpr uint32_t kOffXb = 0;
constexpr uint32_t kOffG = kOffXb + kBStages * 2 * kXbBytes;           // 131072
constexpr uint32_t kOffBar = kOffG + kGStages * 2 * kGBytes;           // 229376
constexpr uint32_t kSmemUsed = kOffBar + 256;
constexpr uint32_t kSmemBytes = kSmemUsed + 1024;                      // + alignment slack
constexpr int kConvThreads = 256;               // warps 0-7
constexpr int kWarpEpi = 8, kWarpG = 12, kWarpMma = 13;
constexpr int kTcThreads = 448;
constexpr uint32_t kTmemCols = 512;
// K-major operands, 128-byte swizzle: row r of a part holds its 64 BF16 k
// values in 128 bytes, 16-byte chunk c stored at chunk c ^ (r % 8); 8-row
// groups 1024 B apart (SBO).  An MMA's K = 16 step starts 32 B further in.
constexpr uint32_t kSbo = 1024;
__host__ __device__ constexpr uint32_t sw128_offset(int row, int chunk) {
    return (uint32_t)(row >> 3) * kSbo + (uint32_t)(row & 7) * 128 + (uint32_t)((chunk ^ (row & 7)) << 4);
}
// kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9, 10-12 = 1), both K-major, N = 256 (bits 17-22: N >> 3),
// M = 128 (bits 24-28: M >> 4)
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTileN >> 3) << 17) |
                            ((uint32_t)(kTileM >> 4) << 24);

// barrier indices (8 bytes each at kOffBar)
enum : int { kBarGFull = 0, kBarGEmpty = 3, kBarConv = 6, kBarBEmpty = 8, kBarAccFull = 10, kBarAccEmpty = 12,
             kBarFin = 14, kNumBars = 15 };
constexpr uint32_t kOffTmemSlot = kOffBar + 8 * kNumBars;              // 4 bytes
constexpr uint32_t kOffAbort = kOffTmemSlot + 4;
static_assert(kOffAbort + 4 <= kSmemUsed, "barrier area");
static_assert(kSmemBytes <= 232448, "227 KB of shared memory per block");

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// One test of the phase; a thread whose phase is not complete is suspended
// (not spinning, so the warps that share its scheduler keep their issue slots)
// until the phase completes or about 0.5 ms pass.
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(500000u)
        : "memory");
    return ok != 0;
}
// Wait for the phase of parity `parity` to complete.  Gives up (false) when
// another role has aborted (if `honor_abort`) or after 4 s, which aborts the CTA.
__device__ __noinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err,
                                       bool honor_abort) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t n = 1;; ++n) {
        if (mbar_test(bar, parity)) return true;
        if ((n & 3u) == 0u) {
            if (honor_abort && *abort_flag) return false;
            if (global_ns() - t0 > 4000000000ull) {
                *abort_flag = 1;
                atomicOr(err, kErrTimeout);
                return false;
            }
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    // start >> 4, LBO (unused with a swizzled K-major layout) = 1, SBO >> 4,
    // descriptor version 1 (bit 46), layout type 2 = 128-byte swizzle (bits 61-63)
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(kSbo >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// (a, b) -> BF16 pairs hi = bf16(x), lo = bf16(x - hi); element a in the low half
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __float22bfloat162_rn(make_float2(a, b));
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __float22bfloat162_rn(make_float2(a - hf.x, b - hf.y));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Waveforms [nwave][K] FP32 -> per (waveform tile, k chunk) 32 KB blocks:
// BF16 hi part then lo part, each 128 rows x 64 k, 128-byte swizzle; rows
// past nwave and k past K are zero.
__global__ void pack_waves_kernel(const float* __restrict__ wave, int nwave, int K, int nk, int n_mtiles,
                                  uint8_t* __restrict__ gpack) {
    const int64_t items = (int64_t)n_mtiles * kTileM * nk * (kKc / 8);   // one item: 8 k of one row
    for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(it % (kKc / 8));
        const int64_t r = it / (kKc / 8);
        const int kc = (int)(r % nk);
        const int m = (int)(r / nk);                 // 0 .. n_mtiles*128 - 1
        const int mt = m / kTileM, ml = m % kTileM;
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int k = kc * kKc + g * 8 + e;
            x[e] = (m < nwave && k < K) ? wave[(size_t)m * K + k] : 0.0f;
        }
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) split2(x[2 * e], x[2 * e + 1], h[e], l[e]);
        uint8_t* blk = gpack + ((size_t)mt * nk + kc) * (2 * kGBytes);
        const uint32_t off = sw128_offset(ml, g);
        *reinterpret_cast<uint4*>(blk + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(blk + kGBytes + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    contract_tc_kernel(const float* __restrict__ pos, int K, const uint8_t* __restrict__ gpack, int64_t nwalk,
                       int nwave, int nk, int n_mpairs, int64_t nunits, double* __restrict__ out, int* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + kOffAbort);
    auto bar = [&](int i) { return sbase + kOffBar + 8u * (uint32_t)i; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGStages; ++s) {
            mbar_init(bar(kBarGFull + s), 1);
            mbar_init(bar(kBarGEmpty + s), 1);
        }
        for (int s = 0; s < kBStages; ++s) {
            mbar_init(bar(kBarConv + s), kConvThreads);
            mbar_init(bar(kBarBEmpty + s), 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(bar(kBarAccFull + s), 1);
            mbar_init(bar(kBarAccEmpty + s), 128);
        }
        mbar_init(bar(kBarFin), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    if (warp == kWarpMma) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(sbase + kOffTmemSlot), "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kOffTmemSlot);

    if (warp == kWarpG) {
        // waveform chunks: pre-split BF16 hi/lo, 32 KB per (waveform tile, k
        // chunk); per position chunk, tile 2 pair then tile 2 pair + 1
        if (lane == 0) {
            int64_t j = 0;
            bool ok = true;
            for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
                const int mp = (int)(u % n_mpairs);
                for (int kc = 0; kc < nk && ok; ++kc) {
                    for (int a = 0; a < 2; ++a, ++j) {
                        const int s = (int)(j % kGStages);
                        if (!(ok = mbar_wait(bar(kBarGEmpty + s), (uint32_t)((j / kGStages) & 1) ^ 1u, abort_flag, err,
                                             true)))
                            break;
                        mbar_arrive_tx(bar(kBarGFull + s), 2 * kGBytes);
                        bulk_load(sbase + kOffG + (uint32_t)s * 2 * kGBytes,
                                  gpack + ((size_t)(2 * mp + a) * nk + kc) * (2 * kGBytes), 2 * kGBytes,
                                  bar(kBarGFull + s));
                    }
                }
            }
            // drain: the last copies issued have landed (or land within the limit)
            for (int64_t jj = j > kGStages ? j - kGStages : 0; jj < j; ++jj)
                mbar_wait(bar(kBarGFull + (int)(jj % kGStages)), (uint32_t)((jj / kGStages) & 1), abort_flag, err, false);
        }
    } else if (warp < kWarpEpi) {
        // converters: FP32 positions -> BF16 hi and lo parts.  A chunk (64 k)
        // is filled in two halves of 32 k; in a half, lane l of converter warp
        // cw converts 8-k group g = l / 8 of walker rows 64 it + 8 cw + l % 8
        // (it = 0..3): a warp reads 8 rows x 128 contiguous bytes, and each
        // 8-lane phase of its 16-byte shared stores covers one chunk of 8
        // rows, which the swizzle spreads over all 32 banks.
        const int ct = threadIdx.x;   // 0 .. kConvThreads - 1
        const int g = (ct >> 3) & 3;
        const int rw = ((ct >> 5) << 3) + (ct & 7);   // row within a 64-row slab
        float4 cur[8], nxt[8];
        auto load = [&](int64_t uu, int kk, int hh, float4(&v)[8]) {
            const int64_t w0 = (uu / n_mpairs) * kTileN;
            const int k = kk * kKc + hh * 32 + g * 8;
#pragma unroll
            for (int it = 0; it < 4; ++it) {
                const int64_t w = w0 + it * 64 + rw;
                const float* p = pos + (size_t)w * K + k;
                const bool in = w < nwalk;
                v[2 * it] = (in && k < K) ? __ldg(reinterpret_cast<const float4*>(p)) : make_float4(0.f, 0.f, 0.f, 0.f);
                v[2 * it + 1] =
                    (in && k + 4 < K) ? __ldg(reinterpret_cast<const float4*>(p + 4)) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        int64_t u = blockIdx.x, i = 0;
        int kc = 0, h = 0;
        if (u < nunits) load(u, 0, 0, cur);
        while (u < nunits) {
            int64_t un = u;
            int kn = kc, hn = h + 1;
            if (hn == 2) {
                hn = 0;
                if (++kn == nk) {
                    kn = 0;
                    un = u + gridDim.x;
                }
            }
            if (un < nunits) load(un, kn, hn, nxt);   // in flight while this half converts
            const int sb = (int)(i % kBStages);
            if (h == 0 &&
                !mbar_wait(bar(kBarBEmpty + sb), (uint32_t)((i / kBStages) & 1) ^ 1u, abort_flag, err, true))
                break;
            uint8_t* xh = sm + kOffXb + (uint32_t)sb * 2 * kXbBytes;
            uint8_t* xl = xh + kXbBytes;
#pragma unroll
            for (int it = 0; it < 4; ++it) {
                const int n = it * 64 + rw;
                const float4 a = cur[2 * it], b = cur[2 * it + 1];
                uint4 hi, lo;
                split2(a.x, a.y, hi.x, lo.x);
                split2(a.z, a.w, hi.y, lo.y);
                split2(b.x, b.y, hi.z, lo.z);
                split2(b.z, b.w, hi.w, lo.w);
                const uint32_t off = sw128_offset(n, h * 4 + g);
                *reinterpret_cast<uint4*>(xh + off) = hi;
                *reinterpret_cast<uint4*>(xl + off) = lo;
            }
            if (h == 1) {
                fence_proxy_async();   // the tensor core reads these through the async proxy
                mbar_arrive(bar(kBarConv + sb));
                ++i;
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) cur[e] = nxt[e];
            u = un;
            kc = kn;
            h = hn;
        }
    } else if (warp == kWarpMma) {
        // MMA issue
        if (lane == 0) {
            int64_t i = 0, j = 0, t = 0;
            bool ok = true;
            for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++t) {
                for (int kc = 0; kc < nk && ok; ++kc, ++i) {
                    const int sb = (int)(i % kBStages);
                    if (!(ok = mbar_wait(bar(kBarConv + sb), (uint32_t)((i / kBStages) & 1), abort_flag, err, true))) break;
                    const uint32_t xa = sbase + kOffXb + (uint32_t)sb * 2 * kXbBytes;
                    for (int a = 0; a < 2; ++a, ++j) {
                        if (kc == 0) {
                            // the epilogue has read this tile's accumulator of the previous unit
                            if (!(ok = mbar_wait(bar(kBarAccEmpty + a), (uint32_t)(t & 1) ^ 1u, abort_flag, err, true)))
                                break;
                        }
                        const int sg = (int)(j % kGStages);
                        if (!(ok = mbar_wait(bar(kBarGFull + sg), (uint32_t)((j / kGStages) & 1), abort_flag, err, true)))
                            break;
                        tc_fence_after();
                        const uint32_t ga = sbase + kOffG + (uint32_t)sg * 2 * kGBytes;
                        const uint32_t d = tmem + (uint32_t)a * kTileN;
#pragma unroll
                        for (int ks = 0; ks < kKc / 16; ++ks) {
                            const uint32_t dk = (uint32_t)ks * 32;        // K = 16 BF16 = 32 B into the rows
                            const uint64_t a_hi = smem_desc(ga + dk), a_lo = smem_desc(ga + kGBytes + dk);
                            const uint64_t b_hi = smem_desc(xa + dk), b_lo = smem_desc(xa + kXbBytes + dk);
                            umma_bf16(d, a_hi, b_hi, (kc > 0 || ks > 0) ? 1u : 0u);
                            umma_bf16(d, a_hi, b_lo, 1u);
                            umma_bf16(d, a_lo, b_hi, 1u);
                        }
                        umma_commit(bar(kBarGEmpty + sg));   // this waveform chunk is free when these are done
                        if (kc == nk - 1) umma_commit(bar(kBarAccFull + a));
                    }
                    if (ok) umma_commit(bar(kBarBEmpty + sb));   // the position chunk too
                }
            }
            // every MMA issued has completed before the tensor memory is freed
            umma_commit(bar(kBarFin));
            mbar_wait(bar(kBarFin), 0, abort_flag, err, false);
        }
    } else {
        // epilogue: warp q reads TMEM lanes 32q .. 32q + 31 (waveform rows)
        const int q = warp - kWarpEpi;   // = warp % 4, the lane quarter this warp may access
        int64_t t = 0;
        bool ok = true;
        for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++t) {
            const int mp = (int)(u % n_mpairs);
            const int64_t n0 = (u / n_mpairs) * kTileN;
            for (int a = 0; a < 2; ++a) {
                if (!(ok = mbar_wait(bar(kBarAccFull + a), (uint32_t)(t & 1), abort_flag, err, true))) break;
                __syncwarp();   // tcgen05.ld is warp-wide
                tc_fence_after();
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)a * kTileN;
                double CS = 0.0, SN = 0.0;
#pragma unroll 1
                for (int c = 0; c < kTileN / 32; ++c) {
                    uint32_t r[32];
                    tmem_ld32(taddr + (uint32_t)c * 32, r);
                    const int64_t nb = n0 + c * 32;
                    // full slices branch-free (32 independent chains the
                    // scheduler can interleave); the last slice masked
                    const int nvalid = (nwalk - nb >= 32) ? 32 : (int)(nwalk - nb);
                    float cs[4] = {0.f, 0.f, 0.f, 0.f}, sn[4] = {0.f, 0.f, 0.f, 0.f};
                    if (nvalid == 32) {
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            float s, co;
                            sincos_reduced(__uint_as_float(r[e]), &s, &co);
                            cs[e & 3] += co;
                            sn[e & 3] += s;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            float s, co;
                            sincos_reduced(__uint_as_float(r[e]), &s, &co);
                            const float m = e < nvalid ? 1.0f : 0.0f;
                            cs[e & 3] = fmaf(m, co, cs[e & 3]);
                            sn[e & 3] = fmaf(m, s, sn[e & 3]);
                        }
                    }
                    CS += (double)((cs[0] + cs[1]) + (cs[2] + cs[3]));
                    SN += (double)((sn[0] + sn[1]) + (sn[2] + sn[3]));
                }
                tc_fence_before();
                mbar_arrive(bar(kBarAccEmpty + a));
                const int jw = (2 * mp + a) * kTileM + q * 32 + lane;
                if (jw < nwave) {
                    atomicAdd(out + 2 * jw, CS);
                    atomicAdd(out + 2 * jw + 1, SN);
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kWarpMma)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Positions already split by the walk (RMS_CONTRACT_BF16X3_PRESPLIT): the same
// pipeline with one TMA warp for the positions in place of the converters.
constexpr int kPsWarpX = 0, kPsWarpG = 1, kPsWarpMma = 2, kPsWarpEpi = 4;
constexpr int kPsThreads = 256;

__global__ void __launch_bounds__(kPsThreads, 1)
    contract_presplit_kernel(const __grid_constant__ CUtensorMap xhi, const __grid_constant__ CUtensorMap xlo,
                             const uint8_t* __restrict__ gpack, int64_t nwalk,
                       int nwave, int nk, int n_mpairs, int64_t nunits, double* __restrict__ out, int* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + kOffAbort);
    auto bar = [&](int i) { return sbase + kOffBar + 8u * (uint32_t)i; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGStages; ++s) {
            mbar_init(bar(kBarGFull + s), 1);
            mbar_init(bar(kBarGEmpty + s), 1);
        }
        for (int s = 0; s < kBStages; ++s) {
            mbar_init(bar(kBarConv + s), 1);   // position chunk landed (TMA)
            mbar_init(bar(kBarBEmpty + s), 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(bar(kBarAccFull + s), 1);
            mbar_init(bar(kBarAccEmpty + s), 128);
        }
        mbar_init(bar(kBarFin), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    if (warp == kPsWarpMma) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(sbase + kOffTmemSlot), "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kOffTmemSlot);

    if (warp == kPsWarpG) {
        // waveform chunks: pre-split BF16 hi/lo, 32 KB per (waveform tile, k
        // chunk); per position chunk, tile 2 pair then tile 2 pair + 1
        if (lane == 0) {
            int64_t j = 0;
            bool ok = true;
            for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
                const int mp = (int)(u % n_mpairs);
                for (int kc = 0; kc < nk && ok; ++kc) {
                    for (int a = 0; a < 2; ++a, ++j) {
                        const int s = (int)(j % kGStages);
                        if (!(ok = mbar_wait(bar(kBarGEmpty + s), (uint32_t)((j / kGStages) & 1) ^ 1u, abort_flag, err,
                                             true)))
                            break;
                        mbar_arrive_tx(bar(kBarGFull + s), 2 * kGBytes);
                        bulk_load(sbase + kOffG + (uint32_t)s * 2 * kGBytes,
                                  gpack + ((size_t)(2 * mp + a) * nk + kc) * (2 * kGBytes), 2 * kGBytes,
                                  bar(kBarGFull + s));
                    }
                }
            }
            // drain: the last copies issued have landed (or land within the limit)
            for (int64_t jj = j > kGStages ? j - kGStages : 0; jj < j; ++jj)
                mbar_wait(bar(kBarGFull + (int)(jj % kGStages)), (uint32_t)((jj / kGStages) & 1), abort_flag, err, false);
        }
    } else if (warp == kPsWarpX) {
        // position chunks: BF16 hi and lo tiles (256 walkers x 64 k), 128-byte
        // swizzle -- the MMA's operand layout, as the walk wrote them
        if (lane == 0) {
            int64_t i = 0;
            bool ok = true;
            for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
                const int y = (int)((u / n_mpairs) * kTileN);
                for (int kc = 0; kc < nk; ++kc, ++i) {
                    const int sb = (int)(i % kBStages);
                    if (!(ok = mbar_wait(bar(kBarBEmpty + sb), (uint32_t)((i / kBStages) & 1) ^ 1u, abort_flag, err, true)))
                        break;
                    const uint32_t dst = sbase + kOffXb + (uint32_t)sb * 2 * kXbBytes;
                    mbar_arrive_tx(bar(kBarConv + sb), 2 * kXbBytes);
                    tma_load_2d(dst, &xhi, kc * kKc, y, bar(kBarConv + sb));
                    tma_load_2d(dst + kXbBytes, &xlo, kc * kKc, y, bar(kBarConv + sb));
                }
            }
            for (int64_t jj = i > kBStages ? i - kBStages : 0; jj < i; ++jj)
                mbar_wait(bar(kBarConv + (int)(jj % kBStages)), (uint32_t)((jj / kBStages) & 1), abort_flag, err, false);
        }
    } else if (warp == kPsWarpMma) {
        // MMA issue
        if (lane == 0) {
            int64_t i = 0, j = 0, t = 0;
            bool ok = true;
            for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++t) {
                for (int kc = 0; kc < nk && ok; ++kc, ++i) {
                    const int sb = (int)(i % kBStages);
                    if (!(ok = mbar_wait(bar(kBarConv + sb), (uint32_t)((i / kBStages) & 1), abort_flag, err, true))) break;
                    const uint32_t xa = sbase + kOffXb + (uint32_t)sb * 2 * kXbBytes;
                    for (int a = 0; a < 2; ++a, ++j) {
                        if (kc == 0) {
                            // the epilogue has read this tile's accumulator of the previous unit
                            if (!(ok = mbar_wait(bar(kBarAccEmpty + a), (uint32_t)(t & 1) ^ 1u, abort_flag, err, true)))
                                break;
                        }
                        const int sg = (int)(j % kGStages);
                        if (!(ok = mbar_wait(bar(kBarGFull + sg), (uint32_t)((j / kGStages) & 1), abort_flag, err, true)))
                            break;
                        tc_fence_after();
                        const uint32_t ga = sbase + kOffG + (uint32_t)sg * 2 * kGBytes;
                        const uint32_t d = tmem + (uint32_t)a * kTileN;
#pragma unroll
                        for (int ks = 0; ks < kKc / 16; ++ks) {
                            const uint32_t dk = (uint32_t)ks * 32;        // K = 16 BF16 = 32 B into the rows
                            const uint64_t a_hi = smem_desc(ga + dk), a_lo = smem_desc(ga + kGBytes + dk);
                            const uint64_t b_hi = smem_desc(xa + dk), b_lo = smem_desc(xa + kXbBytes + dk);
                            umma_bf16(d, a_hi, b_hi, (kc > 0 || ks > 0) ? 1u : 0u);
                            umma_bf16(d, a_hi, b_lo, 1u);
                            umma_bf16(d, a_lo, b_hi, 1u);
                        }
                        umma_commit(bar(kBarGEmpty + sg));   // this waveform chunk is free when these are done
                        if (kc == nk - 1) umma_commit(bar(kBarAccFull + a));
                    }
                    if (ok) umma_commit(bar(kBarBEmpty + sb));   // the position chunk too
                }
            }
            // every MMA issued has completed before the tensor memory is freed
            umma_commit(bar(kBarFin));
            mbar_wait(bar(kBarFin), 0, abort_flag, err, false);
        }
    } else if (warp >= kPsWarpEpi) {
        // epilogue: warp q reads TMEM lanes 32q .. 32q + 31 (waveform rows)
        const int q = warp - kPsWarpEpi;   // = warp % 4, the lane quarter this warp may access
        int64_t t = 0;
        bool ok = true;
        for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++t) {
            const int mp = (int)(u % n_mpairs);
            const int64_t n0 = (u / n_mpairs) * kTileN;
            for (int a = 0; a < 2; ++a) {
                if (!(ok = mbar_wait(bar(kBarAccFull + a), (uint32_t)(t & 1), abort_flag, err, true))) break;
                __syncwarp();   // tcgen05.ld is warp-wide
                tc_fence_after();
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)a * kTileN;
                double CS = 0.0, SN = 0.0;
#pragma unroll 1
                for (int c = 0; c < kTileN / 32; ++c) {
                    uint32_t r[32];
                    tmem_ld32(taddr + (uint32_t)c * 32, r);
                    const int64_t nb = n0 + c * 32;
                    // full slices branch-free (32 independent chains the
                    // scheduler can interleave); the last slice masked
                    const int nvalid = (nwalk - nb >= 32) ? 32 : (int)(nwalk - nb);
                    float cs[4] = {0.f, 0.f, 0.f, 0.f}, sn[4] = {0.f, 0.f, 0.f, 0.f};
                    if (nvalid == 32) {
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            float s, co;
                            sincos_reduced(__uint_as_float(r[e]), &s, &co);
                            cs[e & 3] += co;
                            sn[e & 3] += s;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            float s, co;
                            sincos_reduced(__uint_as_float(r[e]), &s, &co);
                            const float m = e < nvalid ? 1.0f : 0.0f;
                            cs[e & 3] = fmaf(m, co, cs[e & 3]);
                            sn[e & 3] = fmaf(m, s, sn[e & 3]);
                        }
                    }
                    CS += (double)((cs[0] + cs[1]) + (cs[2] + cs[3]));
                    SN += (double)((sn[0] + sn[1]) + (sn[2] + sn[3]));
                }
                tc_fence_before();
                mbar_arrive(bar(kBarAccEmpty + a));
                const int jw = (2 * mp + a) * kTileM + q * 32 + lane;
                if (jw < nwave) {
                    atomicAdd(out + 2 * jw, CS);
                    atomicAdd(out + 2 * jw + 1, SN);
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kPsWarpMma)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// ----------------------------------------------------------------------------
// host side

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// per-device workspace: packed waveforms and the error word
struct Workspace {
    void* p = nullptr;
    size_t bytes = 0;
};
std::mutex g_ws_mu;
std::vector<Workspace> g_ws;

}  // namespace

int contract_phases(const float* d_pos, int64_t nwalk, int nbins, const float* d_wave, int nwave, int method,
                    double* d_out, void* stream, const char** msg, float* kernel_ms) {
    auto fail = [&](int code, const char* m) {
        if (msg) *msg = m;
        return code;
    };
    if (!d_pos || !d_wave || !d_out) return fail(RMS_ERR_ARG, "null buffer");
    if (nwalk < 1 || nbins < 1 || nwave < 1) return fail(RMS_ERR_ARG, "empty contraction");
    if (nbins > (1 << 20) || nwave > (1 << 24)) return fail(RMS_ERR_RANGE, "nbins or nwave too large");
    if (method != RMS_CONTRACT_FP32 && method != RMS_CONTRACT_BF16X3 && method != RMS_CONTRACT_BF16X3_PRESPLIT)
        return fail(RMS_ERR_ARG, "method");
    const int K = 3 * nbins;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(RMS_ERR_CUDA, "cudaGetDevice");
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return fail(RMS_ERR_CUDA, "SM count");
    // kernel time (optional): events around the contraction kernel itself
    struct Events {
        cudaEvent_t a = nullptr, b = nullptr;
        ~Events() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } ev;
    if (kernel_ms && (cudaEventCreate(&ev.a) != cudaSuccess || cudaEventCreate(&ev.b) != cudaSuccess))
        return fail(RMS_ERR_CUDA, "events");
    if (cudaMemsetAsync(d_out, 0, sizeof(double) * 2 * (size_t)nwave, st) != cudaSuccess)
        return fail(RMS_ERR_CUDA, "clearing the output");

    if (method == RMS_CONTRACT_FP32) {
        const int n_mtiles = (nwave + kF32Tile - 1) / kF32Tile;
        const int64_t blocks = (int64_t)n_mtiles * ((nwalk + kF32Tile - 1) / kF32Tile);
        if (blocks > 0x7fffffff) return fail(RMS_ERR_RANGE, "too many walkers");
        if (ev.a) cudaEventRecord(ev.a, st);
        contract_f32_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_pos, nwalk, K, d_wave, nwave, n_mtiles, d_out);
        if (ev.b) cudaEventRecord(ev.b, st);
        if (cudaGetLastError() != cudaSuccess) return fail(RMS_ERR_CUDA, "FP32 contraction launch");
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail(RMS_ERR_CUDA, "FP32 contraction");
    } else {
        const bool presplit = method == RMS_CONTRACT_BF16X3_PRESPLIT;
        if (nbins % 4) return fail(RMS_ERR_ARG, "the tensor-core contraction needs nbins % 4 == 0 (16-byte rows)");
        if (presplit && nbins % 8) return fail(RMS_ERR_ARG, "pre-split positions need nbins % 8 == 0 (16-byte BF16 rows)");
        if (reinterpret_cast<uintptr_t>(d_pos) % 16) return fail(RMS_ERR_ARG, "positions must be 16-byte aligned");
        const int nk = (K + kKc - 1) / kKc;
        const int n_mpairs = (nwave + 2 * kTileM - 1) / (2 * kTileM);
        const int n_mtiles = 2 * n_mpairs;   // the last tiles' rows past nwave are zero
        const size_t gbytes = (size_t)n_mtiles * nk * 2 * kGBytes;
        void* ws;
        {
            std::lock_guard<std::mutex> lk(g_ws_mu);
            if ((int)g_ws.size() <= dev) g_ws.resize(dev + 1);
            Workspace& w = g_ws[dev];
            if (w.bytes < gbytes + 256) {
                if (w.p) cudaFree(w.p);
                w.p = nullptr;
                w.bytes = 0;
                if (cudaMalloc(&w.p, gbytes + 256) != cudaSuccess) return fail(RMS_ERR_NOMEM, "workspace");
                w.bytes = gbytes + 256;
            }
            ws = w.p;
        }
        uint8_t* gpack = static_cast<uint8_t*>(ws);
        int* d_err = reinterpret_cast<int*>(gpack + gbytes);
        if (cudaMemsetAsync(d_err, 0, sizeof(int), st) != cudaSuccess) return fail(RMS_ERR_CUDA, "error word");
        pack_waves_kernel<<<1024, 256, 0, st>>>(d_wave, nwave, K, nk, n_mtiles, gpack);
        if (cudaGetLastError() != cudaSuccess) return fail(RMS_ERR_CUDA, "waveform packing launch");

        static std::once_flag attr_once;
        static cudaError_t attr_err = cudaSuccess;
        std::call_once(attr_once, [] {
            attr_err = cudaFuncSetAttribute(contract_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kSmemBytes);
            if (attr_err == cudaSuccess)
                attr_err = cudaFuncSetAttribute(contract_presplit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kSmemBytes);
        });
        if (attr_err != cudaSuccess) return fail(RMS_ERR_CUDA, "shared memory attribute");
        CUtensorMap mhi, mlo;
        if (presplit) {
            EncodeTiledFn enc = encode_fn();
            if (!enc) return fail(RMS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
            if (nwalk > 0x7fffffffll) return fail(RMS_ERR_RANGE, "too many walkers for one tensor map");
            const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)nwalk};
            const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
            const cuuint32_t box[2] = {(cuuint32_t)kKc, (cuuint32_t)kTileN};
            const cuuint32_t estr[2] = {1, 1};
            uint8_t* hi = reinterpret_cast<uint8_t*>(const_cast<float*>(d_pos));
            uint8_t* lo = hi + (size_t)nwalk * K * 2;
            for (int m = 0; m < 2; ++m)
                if (enc(m ? &mlo : &mhi, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, m ? lo : hi, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                    return fail(RMS_ERR_CUDA, "tensor map of the positions");
        }
        const int64_t nunits = (int64_t)n_mpairs * ((nwalk + kTileN - 1) / kTileN);
        const int grid = (int)std::min<int64_t>(nunits, sms);
        if (ev.a) cudaEventRecord(ev.a, st);
        if (presplit)
            contract_presplit_kernel<<<grid, kPsThreads, kSmemBytes, st>>>(mhi, mlo, gpack, nwalk, nwave, nk, n_mpairs,
                                                                           nunits, d_out, d_err);
        else
            contract_tc_kernel<<<grid, kTcThreads, kSmemBytes, st>>>(d_pos, K, gpack, nwalk, nwave, nk, n_mpairs,
                                                                     nunits, d_out, d_err);
        if (ev.b) cudaEventRecord(ev.b, st);
        if (cudaGetLastError() != cudaSuccess) return fail(RMS_ERR_CUDA, "tensor-core contraction launch");
        int herr = 0;
        if (cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return fail(RMS_ERR_CUDA, "tensor-core contraction");
        if (herr & kErrTimeout) return fail(RMS_ERR_TIMEOUT, "a pipeline wait of the tensor-core contraction ran out");
    }
    if (kernel_ms && (cudaEventElapsedTime(kernel_ms, ev.a, ev.b) != cudaSuccess))
        return fail(RMS_ERR_CUDA, "contraction timing");
    return RMS_OK;
}

}  // namespace rms
