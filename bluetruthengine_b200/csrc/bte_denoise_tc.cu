// bte_denoise_tc.cu -- the denoiser's 3x3 convolution on the 5th-generation
// tensor cores (tcgen05.mma, accumulator in tensor memory).
//
// Implicit GEMM: D[p][co] = sum_{tap, ci} A[p][(tap, ci)] * B[co][(tap, ci)]
// over a CTA tile of 128 consecutive output pixels (flattened n, y, x) and
// all N = Cout output channels (N <= 256, multiple of 16).  The input row of
// pixel p for a tap is gathered from concat(Up ? upsample2x(X1) : X1, X2) at
// the shifted position (zeros outside the image).
//
//   * K advances in stages of one tap x up to 64 channels.  All 128 threads
//     copy the stage's A tile (128 x 64 bf16) and B tile (N x 64 bf16) into
//     shared memory with 16-byte cp.async, in the canonical K-major layout
//     without swizzle: 8-row x 16-byte core matrices, the 16-byte K chunks of
//     a row group LBO bytes apart and consecutive 8-row groups SBO = 128
//     bytes apart.
//   * One thread issues a tcgen05.mma (M = 128, N, K = 16, BF16 in, FP32
//     accumulate) per 16 channels of the stage, then tcgen05.commit to the
//     stage's mbarrier, which releases the buffers for the copy three stages
//     later.
//   * Epilogue: each warp reads its 32 TMEM lanes (= pixels) with
//     tcgen05.ld.32x32b, adds the bias, applies ReLU and stores bf16 rows.
// Every wait is bounded; on a timeout the kernel records an error, stops
// issuing, waits (bounded) for what it issued and frees its tensor memory.
#include "bte_denoise.h"

#include <cuda_bf16.h>

#include <cstdint>

namespace bte {
namespace dn {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kTcM = 128;         // pixels per CTA (TMEM lanes)
constexpr int kTcKStage = 64;     // channels per pipeline stage
constexpr int kTcStages = 3;
constexpr int kTcMaxN = 256;
constexpr int kStageABytes = kTcM * kTcKStage * 2;           // 16 KB
constexpr int kStageBBytes = kTcMaxN * kTcKStage * 2;        // 32 KB
constexpr unsigned kSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity)
{
    for (unsigned i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity));
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    // start >> 4 (bits 0-13), LBO >> 4 (16-29), SBO >> 4 (32-45), version 1 (46-47),
    // base offset 0, LBO mode 0, no swizzle (61-63 = 0)
    return static_cast<uint64_t>((addr >> 4) & 0x3fffu) | (static_cast<uint64_t>((lbo >> 4) & 0x3fffu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, M = 128, N
__device__ __forceinline__ uint32_t instrDesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(kTcM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void ummaCommit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar));
}

template <bool Relu, bool Up>
__global__ void __launch_bounds__(128, 1) kConvTc(const bf16* __restrict__ X1, int C1, const bf16* __restrict__ X2, int C2,
                                                  int N, int H, int W, const bf16* __restrict__ Wk,
                                                  const float* __restrict__ bias, int Cout, bf16* __restrict__ Y,
                                                  unsigned int* errorFlag)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t mbar[kTcStages];
    __shared__ uint32_t tmemBase;
    __shared__ volatile int abortFlag;
    __shared__ volatile int lastCommit;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int Cin = C1 + C2;
    const long long total = static_cast<long long>(N) * H * W;
    const long long p0 = static_cast<long long>(blockIdx.x) * kTcM;
    const uint32_t sA = smemAddr(smem), sB = sA + kTcStages * kStageABytes;
    const uint32_t tmemCols = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : (Cout <= 128 ? 128 : 256));

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemAddr(&tmemBase)),
                     "r"(tmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) mbarInit(smemAddr(&mbar[s]), 1);
        abortFlag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tmem = tmemBase;

    // this thread's A row: pixel p0 + tid
    const long long p = p0 + tid;
    const bool rowValid = p < total;
    const int px = rowValid ? static_cast<int>(p % W) : 0;
    const long long r1 = rowValid ? p / W : 0;
    const int py = static_cast<int>(r1 % H);
    const int pn = static_cast<int>(r1 / H);
    const int chunksPerTap = (Cin + kTcKStage - 1) / kTcKStage;
    const int iters = 9 * chunksPerTap;
    const uint32_t lboA = (kTcM / 8) * 128;          // K chunk stride of the A tile
    const uint32_t lboB = (Cout / 8) * 128;          // K chunk stride of the B tile
    const uint32_t idesc = instrDesc(Cout);

    auto issueCopies = [&](int it) {
        const int stage = it % kTcStages;
        const int tap = it / chunksPerTap;
        const int c0 = (it % chunksPerTap) * kTcKStage;
        const int kc = Cin - c0 < kTcKStage ? Cin - c0 : kTcKStage;
        // A: row tid, kc/8 chunks of 8 channels
        const int yy = py + tap / 3 - 1, xx = px + tap % 3 - 1;
        const bool inImg = rowValid && yy >= 0 && yy < H && xx >= 0 && xx < W;
        const uint32_t aBase = sA + stage * kStageABytes + (tid >> 3) * 128 + (tid & 7) * 16;
        for (int j = 0; j < kc / 8; ++j) {
            const int c = c0 + 8 * j;
            const bf16* src;
            if (c < C1) {
                const int ys = Up ? yy / 2 : yy, xs = Up ? xx / 2 : xx;
                const int Hs = Up ? H / 2 : H, Ws = Up ? W / 2 : W;
                src = X1 + ((static_cast<size_t>(pn) * Hs + (inImg ? ys : 0)) * Ws + (inImg ? xs : 0)) * C1 + c;
            } else {
                src = X2 + ((static_cast<size_t>(pn) * H + (inImg ? yy : 0)) * W + (inImg ? xx : 0)) * C2 + (c - C1);
            }
            cpAsync16(aBase + j * lboA, inImg ? src : X1, inImg);
        }
        // B: Cout rows x kc/8 chunks, spread over the threads
        const int nChunks = Cout * (kc / 8);
        const uint32_t bBase = sB + stage * kStageBBytes;
        for (int e = tid; e < nChunks; e += 128) {
            const int co = e % Cout, j = e / Cout;
            const bf16* src = Wk + (static_cast<size_t>(tap) * Cout + co) * Cin + c0 + 8 * j;
            cpAsync16(bBase + j * lboB + (co >> 3) * 128 + (co & 7) * 16, src, true);
        }
    };

    // All threads run the same barriers whatever happens; a timed-out wait only
    // raises the shared abort flag, after which no copy or MMA is issued.
    if (tid == 0) lastCommit = -1;
    for (int it = 0; it < iters + kTcStages - 1; ++it) {
        if (it < iters && !abortFlag) {
            bool free = true;
            if (it >= kTcStages) {   // the MMAs that read this buffer (stage it - kTcStages) must have finished
                const int prev = it - kTcStages;
                free = mbarWait(smemAddr(&mbar[prev % kTcStages]), static_cast<uint32_t>((prev / kTcStages) & 1));
            }
            if (free) issueCopies(it);
            else abortFlag = 1;
        }
        cpAsyncCommit();
        const int j = it - (kTcStages - 1);
        if (j >= 0 && j < iters) {
            cpAsyncWait<kTcStages - 1>();
            asm volatile("fence.proxy.async.shared::cta;\n" ::);
            __syncthreads();
            if (tid == 0 && !abortFlag) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                const int stage = j % kTcStages;
                const int c0 = (j % chunksPerTap) * kTcKStage;
                const int kc = Cin - c0 < kTcKStage ? Cin - c0 : kTcKStage;
                for (int k = 0; k < kc / 16; ++k) {
                    const uint64_t da = smemDesc(sA + stage * kStageABytes + 2 * k * lboA, lboA, 128);
                    const uint64_t db = smemDesc(sB + stage * kStageBBytes + 2 * k * lboB, lboB, 128);
                    umma(tmem, da, db, idesc, (j > 0 || k > 0) ? 1u : 0u);
                }
                ummaCommit(smemAddr(&mbar[stage]));
                lastCommit = j;
            }
        }
    }
    cpAsyncWait<0>();
    __syncthreads();
    // the last commit covers every MMA issued before it; wait for it (bounded) even after an abort,
    // so that no MMA still writes the tensor memory freed below
    const int last = lastCommit;
    if (last >= 0 && !mbarWait(smemAddr(&mbar[last % kTcStages]), static_cast<uint32_t>((last / kTcStages) & 1)))
        abortFlag = 1;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    __syncthreads();
    if (abortFlag || last != iters - 1) {
        if (tid == 0 && errorFlag) atomicOr(errorFlag, 1u);
    } else {
        // epilogue: warp w owns TMEM lanes 32w..32w+31 = pixels p0 + 32w + lane
        const long long q = p0 + warp * 32 + (tid & 31);
        for (int c = 0; c < Cout; c += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
            if (q < total) {
                uint32_t w8[8];
                for (int k = 0; k < 8; ++k) {
                    float a = __uint_as_float(v[2 * k]) + (bias ? bias[c + 2 * k] : 0.0f);
                    float b = __uint_as_float(v[2 * k + 1]) + (bias ? bias[c + 2 * k + 1] : 0.0f);
                    if (Relu) { a = fmaxf(a, 0.0f); b = fmaxf(b, 0.0f); }
                    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
                    w8[k] = *reinterpret_cast<const uint32_t*>(&h);
                }
                uint4* dst = reinterpret_cast<uint4*>(Y + q * Cout + c);
                dst[0] = make_uint4(w8[0], w8[1], w8[2], w8[3]);
                dst[1] = make_uint4(w8[4], w8[5], w8[6], w8[7]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmemCols));
}


// ---------------------------------------------------------------- row tiles, warp-specialised
// For the full-resolution layers (few channels, many pixels): a tile is 128
// consecutive pixels of one image row.  Its input is the 3-row x 130-pixel
// slab around it (all Cin channels), copied into shared memory once in the
// canonical K-major layout without swizzle: the 16-byte channel chunk j of
// slab row r of input row d at (d * C8 + j) * LBO + 16 r, rows 16 bytes apart.
// The A operand of tap (dy, dx) is then the same slab seen from 16 * dx bytes
// further on (a row shift is a 16-byte address offset), so the nine taps are
// nine descriptors over one copy and nothing is gathered twice.  The layer's
// weights stay in shared memory for the CTA's whole run.
//   warps 0-3   epilogue: tcgen05.ld of TMEM lanes 32w.., bias, ReLU, bf16 stores
//   warps 4-7   producers: cp.async of the next slab, completion signalled to an
//               mbarrier (cp.async.mbarrier.arrive.noinc)
//   warp 8      one thread issues 9 x Cin/16 tcgen05.mma (M = 128, N = Cout, K = 16)
//               per tile and commits them to the slab-free and accumulator-full barriers
// A ring of 2-4 slab buffers (as many as shared memory holds) and two TMEM
// accumulators let copy, MMA and epilogue of consecutive tiles overlap; CTAs
// are persistent over tiles.  The producers walk their chunks with running
// (chunk, slab row, input row) counters, so no division is left in the copy
// loop.  Every wait is bounded: a timeout raises the error flag and stops all
// roles, and the MMA thread waits (bounded) for its last MMAs before the
// tensor memory is freed.
constexpr int kRowPx = 128;
constexpr int kSlabRows = 137;          // 130 used; odd, so chunks of one slab row fall on different banks
constexpr int kSlabLbo = kSlabRows * 16;
constexpr int kRowThreads = 288;
constexpr int kRowMaxStages = 4;
constexpr int kRowSmemBudget = 200 * 1024;
constexpr unsigned kRowSpin = 1u << 24;

__device__ __forceinline__ bool mbarWaitRow(uint32_t bar, uint32_t parity, volatile int* abortFlag)
{
    for (unsigned i = 0; i < kRowSpin; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity));
        if (done) return true;
        if ((i & 1023u) == 1023u && *abortFlag) return false;
    }
    return false;
}

__device__ __forceinline__ void mbarArrive(uint32_t bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(bar));
}

template <bool Relu, bool Up>
__global__ void __launch_bounds__(kRowThreads, 1) kConvTcRow(const bf16* __restrict__ X1, int C1, const bf16* __restrict__ X2,
                                                             int C2, int N, int H, int W, const bf16* __restrict__ Wk,
                                                             const float* __restrict__ bias, int Cout, bf16* __restrict__ Y,
                                                             int stages, unsigned int* errorFlag)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t slabFull[kRowMaxStages], slabEmpty[kRowMaxStages], accFull[2], accEmpty[2];
    __shared__ float sBias[64];
    __shared__ uint32_t tmemBase;
    __shared__ volatile int abortFlag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Cin = C1 + C2, C8 = Cin / 8;
    const int tilesPerRow = (W + kRowPx - 1) / kRowPx;
    const long long numTiles = static_cast<long long>(N) * H * tilesPerRow;
    const uint32_t sW = smemAddr(smem);
    const uint32_t wBytes = 9u * Cout * Cin * 2u;
    const uint32_t slabBytes = 3u * C8 * kSlabLbo;
    const uint32_t sSlab = sW + ((wBytes + 1023u) & ~1023u);
    const uint32_t tmemCols = 2 * Cout <= 32 ? 32 : (2 * Cout <= 64 ? 64 : 128);

    // the layer's weights: tap t, output channel co, chunk j at t * Cout*Cin*2 + j * Cout*16 + co * 16
    for (int e = tid; e < 9 * Cout * C8; e += kRowThreads) {
        const int j = e % C8, co = (e / C8) % Cout, t = e / (C8 * Cout);
        cpAsync16(sW + t * Cout * Cin * 2 + j * Cout * 16 + co * 16, Wk + (static_cast<size_t>(t) * Cout + co) * Cin + 8 * j, true);
    }
    cpAsyncCommit();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemAddr(&tmemBase)),
                     "r"(tmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid < Cout) sBias[tid] = bias ? bias[tid] : 0.0f;
    if (tid == 0) {
        for (int b = 0; b < stages; ++b) {
            mbarInit(smemAddr(&slabFull[b]), 128);
            mbarInit(smemAddr(&slabEmpty[b]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbarInit(smemAddr(&accFull[b]), 1);
            mbarInit(smemAddr(&accEmpty[b]), 4);
        }
        abortFlag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    cpAsyncWait<0>();
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tmem = tmemBase;
    const long long first = blockIdx.x, stride = gridDim.x;
    const int local = first < numTiles ? static_cast<int>((numTiles - first + stride - 1) / stride) : 0;
    auto tileOf = [&](int i, int& n, int& y, int& x0) {
        const long long t = first + static_cast<long long>(i) * stride;
        x0 = static_cast<int>(t % tilesPerRow) * kRowPx;
        const long long r = t / tilesPerRow;
        y = static_cast<int>(r % H);
        n = static_cast<int>(r / H);
    };

    if (warp >= 4 && warp < 8) {   // ---- producers
        // chunk e = pt + 128 k of the slab is (input row d, slab row r, channel chunk j) with
        // e = (d * 130 + r) * C8 + j; stepping e by 128 steps (r, j) by (128 / C8, 128 % C8)
        const int pt = tid - 128, J1 = C1 / 8, total = 3 * 130 * C8;
        const int stepJ = 128 % C8, stepR = 128 / C8, j0 = pt % C8, r0 = pt / C8;
        const int Hs = Up ? H / 2 : H, Ws = Up ? W / 2 : W;
        int b = 0, round = 0;
        for (int i = 0; i < local && !abortFlag; ++i) {
            if (round > 0 && !mbarWaitRow(smemAddr(&slabEmpty[b]), static_cast<uint32_t>((round - 1) & 1), &abortFlag)) {
                abortFlag = 1;
                break;
            }
            int n, y, x0;
            tileOf(i, n, y, x0);
            const uint32_t slab = sSlab + b * slabBytes;
            // element offsets of input row y - 1 + d in X1 (at its own resolution) and X2
            long long o1 = 0, o2 = 0;
            bool rowIn = false;
            auto rowSetup = [&](int d) {
                const int yy = y - 1 + d;
                rowIn = yy >= 0 && yy < H;
                o1 = ((static_cast<long long>(n) * Hs + (Up ? (yy >> 1) : yy)) * Ws) * C1;
                o2 = ((static_cast<long long>(n) * H + yy) * W) * C2;
            };
            int j = j0, r = r0, d = 0;
            rowSetup(0);
            for (int e = pt; e < total; e += 128) {
                const int xx = x0 - 1 + r;
                const bool inImg = rowIn && xx >= 0 && xx < W;
                const bf16* src = X1;
                if (inImg)
                    src = j < J1 ? X1 + o1 + static_cast<long long>(Up ? (xx >> 1) : xx) * C1 + 8 * j
                                 : X2 + o2 + static_cast<long long>(xx) * C2 + 8 * (j - J1);
                cpAsync16(slab + (d * C8 + j) * kSlabLbo + r * 16, src, inImg);
                j += stepJ;
                r += stepR;
                if (j >= C8) { j -= C8; ++r; }
                if (r >= 130) { r -= 130; ++d; rowSetup(d); }
            }
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smemAddr(&slabFull[b])));
            if (++b == stages) { b = 0; ++round; }
        }
        cpAsyncWait<0>();
    } else if (warp == 8) {   // ---- MMA issue
        if (lane == 0) {
            const uint32_t idesc = instrDesc(Cout);
            const uint32_t lboB = Cout * 16;
            int issued = -1, b = 0, round = 0;
            for (int i = 0; i < local && !abortFlag; ++i) {
                if (!mbarWaitRow(smemAddr(&slabFull[b]), static_cast<uint32_t>(round & 1), &abortFlag) ||
                    (i >= 2 && !mbarWaitRow(smemAddr(&accEmpty[i & 1]), static_cast<uint32_t>(((i - 2) >> 1) & 1), &abortFlag))) {
                    abortFlag = 1;
                    break;
                }
                asm volatile("fence.proxy.async.shared::cta;\n" ::);
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                const uint32_t slab = sSlab + b * slabBytes;
                const uint32_t acc = tmem + static_cast<uint32_t>((i & 1) * Cout);
                for (int t = 0; t < 9; ++t) {
                    const int dy = t / 3, dx = t % 3;
                    for (int kk = 0; kk < Cin / 16; ++kk) {
                        const uint64_t da = smemDesc(slab + (dy * C8 + 2 * kk) * kSlabLbo + dx * 16, kSlabLbo, 128);
                        const uint64_t db = smemDesc(sW + t * Cout * Cin * 2 + 2 * kk * lboB, lboB, 128);
                        umma(acc, da, db, idesc, (t > 0 || kk > 0) ? 1u : 0u);
                    }
                }
                ummaCommit(smemAddr(&slabEmpty[b]));
                ummaCommit(smemAddr(&accFull[i & 1]));
                issued = i;
                if (++b == stages) { b = 0; ++round; }
            }
            // whatever happened, the last MMAs must be done before the tensor memory is freed
            if (issued >= 0 && !mbarWaitRow(smemAddr(&accFull[issued & 1]), static_cast<uint32_t>((issued >> 1) & 1), &abortFlag)) {
                for (unsigned s = 0; s < kRowSpin; ++s) {   // on abort, wait on (bounded) without the abort exit
                    uint32_t done;
                    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                                 : "=r"(done)
                                 : "r"(smemAddr(&accFull[issued & 1])), "r"(static_cast<uint32_t>((issued >> 1) & 1)));
                    if (done) break;
                }
            }
        }
    } else {   // ---- epilogue, warps 0-3: TMEM lanes 32w..32w+31 = tile pixels 32w..32w+31
        for (int i = 0; i < local && !abortFlag; ++i) {
            const int a = i & 1;
            if (!mbarWaitRow(smemAddr(&accFull[a]), static_cast<uint32_t>((i >> 1) & 1), &abortFlag)) {
                abortFlag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            int n, y, x0;
            tileOf(i, n, y, x0);
            const int x = x0 + warp * 32 + lane;
            for (int c = 0; c < Cout; c += 16) {
                uint32_t v[16];
                const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(a * Cout + c);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                               "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                             : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
                if (x < W) {
                    uint32_t w8[8];
                    for (int k = 0; k < 8; ++k) {
                        float p = __uint_as_float(v[2 * k]) + sBias[c + 2 * k];
                        float q = __uint_as_float(v[2 * k + 1]) + sBias[c + 2 * k + 1];
                        if (Relu) { p = fmaxf(p, 0.0f); q = fmaxf(q, 0.0f); }
                        const __nv_bfloat162 h = __floats2bfloat162_rn(p, q);
                        w8[k] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(Y + ((static_cast<size_t>(n) * H + y) * W + x) * Cout + c);
                    dst[0] = make_uint4(w8[0], w8[1], w8[2], w8[3]);
                    dst[1] = make_uint4(w8[4], w8[5], w8[6], w8[7]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
            __syncwarp();
            if (lane == 0) mbarArrive(smemAddr(&accEmpty[a]));
        }
    }
    __syncthreads();
    if (abortFlag && tid == 0 && errorFlag) atomicOr(errorFlag, 1u);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmemCols));
}

}  // namespace

constexpr int kTcSmem = kTcStages * (kStageABytes + kStageBBytes);

bool convTcSupported(int Cin, int Cout) { return Cout % 16 == 0 && Cout >= 16 && Cout <= kTcMaxN && Cin % 16 == 0; }

void conv3x3Tc(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
               const float* bias, int Cout, bool relu, void* Y, unsigned int* errorFlag, cudaStream_t st)
{
    const long long total = static_cast<long long>(N) * H * W;
    const unsigned grid = static_cast<unsigned>((total + kTcM - 1) / kTcM);
    static bool attrSet = false;
    if (!attrSet) {
        cudaFuncSetAttribute(kConvTc<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        cudaFuncSetAttribute(kConvTc<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        cudaFuncSetAttribute(kConvTc<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        cudaFuncSetAttribute(kConvTc<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        attrSet = true;
    }
    auto launch = [&](auto kernel) {
        kernel<<<grid, 128, kTcSmem, st>>>(static_cast<const bf16*>(X1), C1, static_cast<const bf16*>(X2), C2, N, H, W,
                                           static_cast<const bf16*>(Wk), bias, Cout, static_cast<bf16*>(Y), errorFlag);
    };
    if (relu) {
        if (up) launch(kConvTc<true, true>);
        else launch(kConvTc<true, false>);
    } else {
        if (up) launch(kConvTc<false, true>);
        else launch(kConvTc<false, false>);
    }
}

// slab buffers that fit beside the layer's weights (at most kRowMaxStages; fewer than 2 = unsupported)
int convTcRowStages(int Cin, int Cout)
{
    const long long w = (9LL * Cout * Cin * 2 + 1023) & ~1023LL, slab = 3LL * (Cin / 8) * kSlabLbo;
    const long long fit = (kRowSmemBudget - w) / slab;
    return static_cast<int>(fit < kRowMaxStages ? fit : kRowMaxStages);
}

int convTcRowSmem(int Cin, int Cout)
{
    return static_cast<int>(((9LL * Cout * Cin * 2 + 1023) & ~1023LL) + convTcRowStages(Cin, Cout) * 3LL * (Cin / 8) * kSlabLbo);
}

bool convTcRowSupported(int C1, int C2, int Cout)
{
    const int Cin = C1 + C2;
    return (Cout == 16 || Cout == 32 || Cout == 48 || Cout == 64) && Cin % 16 == 0 && C1 % 8 == 0 && Cin >= 16 &&
           convTcRowStages(Cin, Cout) >= 2;
}

void conv3x3TcRow(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
                  const float* bias, int Cout, bool relu, void* Y, unsigned int* errorFlag, cudaStream_t st)
{
    const int smemBytes = convTcRowSmem(C1 + C2, Cout), stages = convTcRowStages(C1 + C2, Cout);
    auto launch = [&](auto kernel) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smemBytes);
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kRowThreads, smemBytes) != cudaSuccess || per < 1) per = 1;
        const int tmemCols = 2 * Cout <= 32 ? 32 : (2 * Cout <= 64 ? 64 : 128);
        if (per * tmemCols > 512) per = 512 / tmemCols;   // every resident CTA gets its tensor memory at once
        const long long tiles = static_cast<long long>(N) * H * ((W + kRowPx - 1) / kRowPx);
        const long long grid = tiles < static_cast<long long>(sms) * per ? tiles : static_cast<long long>(sms) * per;
        kernel<<<static_cast<unsigned>(grid), kRowThreads, smemBytes, st>>>(
            static_cast<const bf16*>(X1), C1, static_cast<const bf16*>(X2), C2, N, H, W, static_cast<const bf16*>(Wk), bias,
            Cout, static_cast<bf16*>(Y), stages, errorFlag);
    };
    if (relu) {
        if (up) launch(kConvTcRow<true, true>);
        else launch(kConvTcRow<true, false>);
    } else {
        if (up) launch(kConvTcRow<false, true>);
        else launch(kConvTcRow<false, false>);
    }
}

}  // namespace dn
}  // namespace bte
