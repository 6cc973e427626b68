// bte_denoise_tc.cu -- the denoiser's 3x3 convolution on the 5th-generation
// tensor cores (tcgen05.mma, accumulator in tensor memory).  Two kernels:
// kConvTcRow (the default, further below: persistent, warp-specialised, row
// tiles fed by TMA, weights resident) and kConvTc, the first version described
// here (pixel tiles, operands gathered per tile by cp.async).
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

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

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
// A pipeline wait that lasts this long has failed (a stage waits microseconds): the waits below give up after
// this much time, or after their iteration limit, whichever comes first, and the kernel reports an error.
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ unsigned long long globalNs()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// true once kWaitNs have passed since the first call of a wait (t0 starts at 0)
__device__ __forceinline__ bool waitExpired(unsigned long long& t0)
{
    const unsigned long long t = globalNs();
    if (t0 == 0) { t0 = t; return false; }
    return t - t0 > kWaitNs;
}

__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0));
}
// the copy without the source-size operand (no zero fill): for chunks known to be in range
__device__ __forceinline__ void cpAsync16Full(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}
__device__ __forceinline__ void stSharedZero16(uint32_t dst)
{
    asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};\n" ::"r"(dst), "r"(0u));
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
    unsigned long long t0 = 0;
    for (unsigned i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity));
        if (done) return true;
        if ((i & 1023u) == 1023u && waitExpired(t0)) return false;
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
            // load and wait in one statement, so that no use of v is scheduled before the wait
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr));
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
// For every layer with enough pixels: a tile is 128 consecutive pixels of R
// consecutive image rows (R = 1, 2 or 4 by the layer's size).  Its input is
// the (R + 2)-row x 130-pixel slab around it (the pass's input channels),
// staged in shared memory once in the
// canonical K-major layout with 32-byte swizzling: block jb of 16 channels
// holds slab pixel r of input row d as one 32-byte row at
// jb * kSlabJStride + (d * 130 + r) * 32, its two 16-byte halves exchanged
// when bit 7 of the address is set.  The A operand of tap (dy, dx) is the
// same block seen from (dy * 130 + dx) * 32 bytes on (a pixel shift is one
// row), so the nine taps are nine descriptors over one copy.  The layer's
// weights stay in shared memory for the CTA's whole run.
//   producers   blocks read in place (X2, and X1 unless it is upsampled) come
//               by TMA: one cp.async.bulk.tensor per block, a box of 16
//               channels x 130 pixels x R + 2 rows (32-byte rows, the copy
//               engine swizzles and fills the out-of-image part with zeros),
//               issued by one thread (lane 0 of warp 9).  With an upsampled X1
//               (layers that run in passes) warps 4-7 produce instead: X1 comes
//               by TMA at its own resolution (16 channels x 66 pixels x R + 1
//               rows per block, one tile ahead, into a double-buffered staging
//               area) and their 128 threads expand it into the slab with
//               16-byte shared-memory copies, walking running counters.
//   warp 8      one thread issues R x 9 x Cin/16 tcgen05.mma (M = 128, N =
//               Cout, K = 16) per tile, fully unrolled (Cin/16 and R are
//               template parameters) so that every descriptor is a base plus a
//               constant: small MMAs are bound by their issue rate, and a
//               runtime loop around them costs up to three times the issue
//               time.  The MMAs are committed to the slab-free and
//               accumulator-full barriers.
//   epilogue    warps 0-7 (0-3 with an upsampled X1): tcgen05.ld of the TMEM
//               lanes of warp w % 4, each of a pair of warps taking half of the
//               output channels; the accumulator is released once read; bias,
//               ReLU, bf16 stores (or FP32 partial sums), and the fused pool.
// A ring of 2-4 slab buffers (as many as shared memory holds) and a ring of
// 2-4 TMEM accumulators let copy, MMA and epilogue of consecutive tiles
// overlap; CTAs are persistent over tiles.  Every wait is bounded: a timeout
// raises the error flag and stops all roles, and the MMA thread waits
// (bounded) for its last MMAs before the tensor memory is freed.
constexpr int kRowPx = 128;
constexpr int kSlabPx = kRowPx + 2;
constexpr int kSlabDStride = kSlabPx * 32;                          // 4160: one input row of one 16-channel block
constexpr int kStgPx = kRowPx / 2 + 2;                              // 66 source pixels of an upsampled input
constexpr int kStgDStride = kStgPx * 32;                            // 2112: one source row of one block
// A tile covers R output rows (1, 2 or 4): its slab holds R + 2 input rows, an upsampled input's staging R + 1
// source rows; blocks are swizzle-atom (256-byte) aligned
__host__ __device__ constexpr int slabJStride(int R) { return ((R + 2) * kSlabDStride + 255) / 256 * 256; }
__host__ __device__ constexpr int stgJStride(int R) { return ((R + 1) * kStgDStride + 255) / 256 * 256; }
constexpr int kRowThreads = 320;   // 10 warps: 0-7 epilogue / producers, 8 MMA, 9 TMA
constexpr int kRowMaxStages = 4;
constexpr int kRowMaxAccs = 4;
constexpr int kRowSmemBudget = 218 * 1024;
constexpr int kRowMaxK16 = 6;           // Cin up to 96 per pass
constexpr int kRowMaxCout = 128;
constexpr unsigned kRowSpin = 1u << 24;

__device__ __forceinline__ bool mbarWaitRow(uint32_t bar, uint32_t parity, volatile int* abortFlag)
{
    unsigned long long t0 = 0;
    for (unsigned i = 0; i < kRowSpin; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity));
        if (done) return true;
        if ((i & 1023u) == 1023u && (*abortFlag || waitExpired(t0))) return false;
    }
    return false;
}

// A wait that nothing completes: one warp initialises an mbarrier that no thread arrives at and waits on its
// first phase with the row-tile kernel's bounded wait.  The wait must give up (status 2) in about kWaitNs
// instead of hanging; status 1 would mean it returned as if completed.  Elapsed time in ns to *ns.
__global__ void kWaitTimeoutProbe(unsigned int* status, unsigned long long* ns)
{
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abortFlag;
    if (threadIdx.x == 0) {
        mbarInit(smemAddr(&bar), 1);
        abortFlag = 0;
    }
    __syncthreads();
    const unsigned long long t0 = globalNs();
    const bool done = mbarWaitRow(smemAddr(&bar), 0u, &abortFlag);
    const unsigned long long t1 = globalNs();
    if (threadIdx.x == 0) {
        *status = done ? 1u : 2u;
        *ns = t1 - t0;
    }
}

__device__ __forceinline__ void mbarArrive(uint32_t bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(bar));
}

// 32-byte swizzle (the TMA's CU_TENSOR_MAP_SWIZZLE_32B and the MMA's 32B layout): the 16-byte half of a
// 32-byte row is exchanged when address bit 7 is set
__device__ __forceinline__ uint32_t sw32(uint32_t addr) { return addr ^ ((addr >> 3) & 16u); }

// K-major 32-byte-swizzled operand: rows of 32 bytes, 8-row groups 256 bytes apart
__device__ __forceinline__ uint64_t smemDescSw32(uint32_t addr)
{
    return smemDesc(addr, 16, 256) | (6ull << 61);
}

__device__ __forceinline__ uint4 ldShared16(uint32_t addr)
{
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr));
    return v;
}

__device__ __forceinline__ void stShared16(uint32_t addr, uint4 v)
{
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w));
}

// Cout (8, 16, 24, 32, 48, 64, 96 or 128) consecutive 32-bit TMEM columns of the warp's 32 lanes into v, and the
// wait for them inside the same asm statement: the registers are defined only once the wait has returned, so
// the compiler cannot schedule a use of v between the load and the wait
template <int NV>
__device__ __forceinline__ void tmemLoadWait(uint32_t taddr, int Cout, uint32_t (&v)[NV])
{
    switch (Cout) {
        case 8:
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                         : "r"(taddr));
            break;
        case 24:
            if constexpr (NV >= 24) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%24];\n"
                         "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16,%17,%18,%19,%20,%21,%22,%23}, [%25];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                           "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23])
                         : "r"(taddr), "r"(taddr + 16u));
            }
            break;
        case 16:
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr + 0u));
            break;
        case 32:
            if constexpr (NV >= 32) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                           "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                           "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                           "=r"(v[30]), "=r"(v[31])
                         : "r"(taddr + 0u));
            }
            break;
        case 48:
            if constexpr (NV >= 48) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%48];\n"
                         "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, [%49];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                           "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                           "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                           "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]),
                           "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]),
                           "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47])
                         : "r"(taddr + 0u), "r"(taddr + 32u));
            }
            break;
        case 64:
            if constexpr (NV >= 64) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                           "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                           "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                           "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]),
                           "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]),
                           "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
                           "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]),
                           "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]),
                           "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
                         : "r"(taddr + 0u));
            }
            break;
        case 96:
            if constexpr (NV >= 96) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%96];\n"
                         "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%64,%65,%66,%67,%68,%69,%70,%71,%72,%73,%74,%75,%76,%77,%78,%79,%80,%81,%82,%83,%84,%85,%86,%87,%88,%89,%90,%91,%92,%93,%94,%95}, [%97];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                           "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                           "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                           "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]),
                           "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]),
                           "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
                           "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]),
                           "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]),
                           "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63]), "=r"(v[64]), "=r"(v[65]),
                           "=r"(v[66]), "=r"(v[67]), "=r"(v[68]), "=r"(v[69]), "=r"(v[70]), "=r"(v[71]),
                           "=r"(v[72]), "=r"(v[73]), "=r"(v[74]), "=r"(v[75]), "=r"(v[76]), "=r"(v[77]),
                           "=r"(v[78]), "=r"(v[79]), "=r"(v[80]), "=r"(v[81]), "=r"(v[82]), "=r"(v[83]),
                           "=r"(v[84]), "=r"(v[85]), "=r"(v[86]), "=r"(v[87]), "=r"(v[88]), "=r"(v[89]),
                           "=r"(v[90]), "=r"(v[91]), "=r"(v[92]), "=r"(v[93]), "=r"(v[94]), "=r"(v[95])
                         : "r"(taddr + 0u), "r"(taddr + 64u));
            }
            break;
        case 128:
            if constexpr (NV >= 128) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x128.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63,%64,%65,%66,%67,%68,%69,%70,%71,%72,%73,%74,%75,%76,%77,%78,%79,%80,%81,%82,%83,%84,%85,%86,%87,%88,%89,%90,%91,%92,%93,%94,%95,%96,%97,%98,%99,%100,%101,%102,%103,%104,%105,%106,%107,%108,%109,%110,%111,%112,%113,%114,%115,%116,%117,%118,%119,%120,%121,%122,%123,%124,%125,%126,%127}, [%128];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                           "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                           "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                           "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]),
                           "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]),
                           "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
                           "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]),
                           "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]),
                           "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63]), "=r"(v[64]), "=r"(v[65]),
                           "=r"(v[66]), "=r"(v[67]), "=r"(v[68]), "=r"(v[69]), "=r"(v[70]), "=r"(v[71]),
                           "=r"(v[72]), "=r"(v[73]), "=r"(v[74]), "=r"(v[75]), "=r"(v[76]), "=r"(v[77]),
                           "=r"(v[78]), "=r"(v[79]), "=r"(v[80]), "=r"(v[81]), "=r"(v[82]), "=r"(v[83]),
                           "=r"(v[84]), "=r"(v[85]), "=r"(v[86]), "=r"(v[87]), "=r"(v[88]), "=r"(v[89]),
                           "=r"(v[90]), "=r"(v[91]), "=r"(v[92]), "=r"(v[93]), "=r"(v[94]), "=r"(v[95]),
                           "=r"(v[96]), "=r"(v[97]), "=r"(v[98]), "=r"(v[99]), "=r"(v[100]), "=r"(v[101]),
                           "=r"(v[102]), "=r"(v[103]), "=r"(v[104]), "=r"(v[105]), "=r"(v[106]), "=r"(v[107]),
                           "=r"(v[108]), "=r"(v[109]), "=r"(v[110]), "=r"(v[111]), "=r"(v[112]), "=r"(v[113]),
                           "=r"(v[114]), "=r"(v[115]), "=r"(v[116]), "=r"(v[117]), "=r"(v[118]), "=r"(v[119]),
                           "=r"(v[120]), "=r"(v[121]), "=r"(v[122]), "=r"(v[123]), "=r"(v[124]), "=r"(v[125]),
                           "=r"(v[126]), "=r"(v[127])
                         : "r"(taddr + 0u));
            }
            break;
        default: break;
    }
}

__device__ __forceinline__ void mbarArriveExpectTx(uint32_t bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(bar), "r"(bytes));
}

// one box (8 channels x pixels x rows) of an NHWC bf16 tensor into shared memory (no multicast)
__device__ __forceinline__ void tmaLoadBox(uint32_t dst, const CUtensorMap* map, int c, int x, int y, int n, uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                 ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(x), "r"(y), "r"(n), "r"(bar)
                 : "memory");
}

// output row r of the tile (accumulator at acc + r * Cout columns): the nine taps x K16 k-steps, descriptors
// as constant offsets from the tile's bases (tap (dy, dx) reads slab row r + dy from pixel dx on)
template <int K16, int R>
__device__ __forceinline__ void issueRowTile(uint32_t acc, uint32_t Cout, uint64_t aDesc0, uint64_t bDesc0, uint32_t bStep,
                                             uint32_t idesc)
{
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int t = 0; t < 9; ++t) {
#pragma unroll
            for (int kk = 0; kk < K16; ++kk) {
                const uint64_t da =
                    aDesc0 + static_cast<uint32_t>(((r + t / 3) * kSlabDStride + (t % 3) * 32 + kk * slabJStride(R)) / 16);
                const uint64_t db = bDesc0 + static_cast<uint32_t>(t * K16 + kk) * bStep;
                umma(acc + r * Cout, da, db, idesc, (t > 0 || kk > 0) ? 1u : 0u);
            }
        }
    }
}

// One pass of a layer whose weights and slabs do not fit shared memory at once: the input channels
// [c1lo, c1lo + C1) of X1 and [c2lo, c2lo + C2) of X2, weight columns [wOff, wOff + C1 + C2) of rows
// wStride long.  partIn (FP32, may alias partOut) is added to the accumulator; with partOut the sum is
// stored there in FP32, otherwise bias and ReLU follow and Y receives bf16.  The partial sums are private
// to the passes and laid out per 128-pixel row segment, channel-major inside it:
// [(n * H + y) * tilesPerRow + x / 128][Cout][128], so a warp's 32 pixels of one channel are 128
// contiguous bytes.  With pool (two output rows per tile, even H and W) the epilogue also writes the
// 2x2 average of the bf16 outputs, summed in the order (y, x), (y, x + 1), (y + 1, x), (y + 1, x + 1) as the
// separate pooling kernel does.
struct RowPass {
    int c1lo, c2lo, wStride, wOff;
    const float* partIn;
    float* partOut;
    bf16* pool;   // two-row tiles of the last pass: also the 2x2 average pool of Y ([N][H/2][W/2][Cout]), or null
};

template <bool Relu, bool Up, int K16, int R>
__global__ void __launch_bounds__(kRowThreads, 1) kConvTcRow(const __grid_constant__ CUtensorMap mapX1,
                                                             const __grid_constant__ CUtensorMap mapX2,
                                                             int C1, int C2, int N, int H, int W,
                                                             const bf16* __restrict__ Wk, const float* __restrict__ bias,
                                                             int Cout, bf16* __restrict__ Y, RowPass pass, int stages,
                                                             int accs, int tmemCols, unsigned int* errorFlag)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t slabFull[kRowMaxStages], slabEmpty[kRowMaxStages], accFull[kRowMaxAccs], accEmpty[kRowMaxAccs];
    __shared__ uint64_t stgFull[2], stgEmpty[2];
    __shared__ float sBias[kRowMaxCout];
    __shared__ uint32_t tmemBase;
    __shared__ volatile int abortFlag;
    // programmatic dependent launch: the next convolution may start its prologue (weights, barriers, tensor
    // memory) as soon as SMs free up; everything that reads or writes activations waits for this grid below
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Cin = 16 * K16, C8 = Cin / 8, J1 = C1 / 16;   // Cin = C1 + C2 (multiples of 16), checked by the launcher
    const int cpJ = Up ? J1 : 0;   // blocks [0, cpJ) expanded from the staging area, [cpJ, K16) by TMA
    constexpr int JS = slabJStride(R), SJS = stgJStride(R);
    const int tilesPerRow = (W + kRowPx - 1) / kRowPx, rowTiles = (H + R - 1) / R;
    const int numTiles = N * rowTiles * tilesPerRow;   // < 2^31, checked by the launcher
    const uint32_t sW = smemAddr(smem);
    const uint32_t wBytes = 9u * Cout * Cin * 2u;
    const uint32_t slabBytes = static_cast<uint32_t>(K16) * JS;
    const uint32_t sSlab = sW + ((wBytes + 1023u) & ~1023u);
    const uint32_t sStg = sSlab + stages * slabBytes, stgBytes = static_cast<uint32_t>(J1) * SJS;
    if (sW & 1023u) {   // TMA boxes need 128-byte aligned destinations; the layout assumes a 1024-byte aligned base
        if (tid == 0 && errorFlag) atomicOr(errorFlag, 1u);
        return;
    }

    // the pass's weights: tap t, output channel co, chunk j at t * Cout*Cin*2 + j * Cout*16 + co * 16
    for (int e = tid; e < 9 * Cout * C8; e += kRowThreads) {
        const int j = e % C8, co = (e / C8) % Cout, t = e / (C8 * Cout);
        cpAsync16(sW + t * Cout * Cin * 2 + j * Cout * 16 + co * 16,
                  Wk + (static_cast<size_t>(t) * Cout + co) * pass.wStride + pass.wOff + 8 * j, true);
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
            // upsampled input: 128 expanding producer threads + the TMA thread's expect-tx arrival; else the latter only
            mbarInit(smemAddr(&slabFull[b]), Up ? 129 : 1);
            mbarInit(smemAddr(&slabEmpty[b]), 1);
        }
        for (int b = 0; b < accs; ++b) {
            mbarInit(smemAddr(&accFull[b]), 1);
            mbarInit(smemAddr(&accEmpty[b]), Up ? 4 : 8);   // one arrival per epilogue warp
        }
        for (int b = 0; b < 2; ++b) {
            mbarInit(smemAddr(&stgFull[b]), 1);
            mbarInit(smemAddr(&stgEmpty[b]), 128);
        }
        abortFlag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    cpAsyncWait<0>();
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    // the previous kernel in the stream (its activations, partial sums) has completed past this point; only
    // the weights and bias, which no kernel in flight writes, were read before it
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    const uint32_t tmem = tmemBase;
    const int first = blockIdx.x, stride = gridDim.x;
    const int local = first < numTiles ? (numTiles - first + stride - 1) / stride : 0;
    auto tileOf = [&](int i, int& n, int& y, int& x0) {   // y: the tile's first output row
        const unsigned t = static_cast<unsigned>(first + i * stride), r = t / tilesPerRow;
        x0 = static_cast<int>(t - r * tilesPerRow) * kRowPx;
        y = static_cast<int>(r % static_cast<unsigned>(rowTiles)) * R;
        n = static_cast<int>(r / static_cast<unsigned>(rowTiles));
    };

    // roles: upsampled input -- warps 4-7 produce (TMA by thread 128, expansion by all), warps 0-3 epilogue;
    // otherwise -- lane 0 of warp 9 produces (TMA), warps 0-7 epilogue (two per TMEM lane group, each taking
    // half of the output channels); warp 8 issues the MMAs
    const bool producer = Up ? (warp >= 4 && warp < 8) : (warp == 9 && lane == 0);
    const bool epilogue = Up ? warp < 4 : warp < 8;
    if (producer) {   // ---- producers
        // expanded 16-byte unit e = pt + 128 k is (input row d, block j, slab pixel r, half h) with
        // e = ((d * cpJ + j) * 130 + r) * 2 + h: a warp copies 16 consecutive pixels of one block
        const int pt = Up ? tid - 128 : 0, total = (R + 2) * kSlabPx * cpJ * 2, h = pt & 1;
        const uint32_t txBytes = static_cast<uint32_t>(K16 - cpJ) * (R + 2u) * kSlabDStride;
        // staging TMA of local tile ii (upsampled input at its own resolution) into buffer ii & 1
        auto issueStage = [&](int ii) {
            int n2, y2, x2;
            tileOf(ii, n2, y2, x2);
            const uint32_t dst = sStg + (ii & 1) * stgBytes, bar = smemAddr(&stgFull[ii & 1]);
            mbarArriveExpectTx(bar, static_cast<uint32_t>(J1) * (R + 1u) * kStgDStride);
            for (int j = 0; j < J1; ++j)
                tmaLoadBox(dst + j * SJS, &mapX1, pass.c1lo + 16 * j, (x2 - 1) >> 1, (y2 - 1) >> 1, n2, bar);
        };
        if (Up && pt == 0 && local > 0) issueStage(0);
        int b = 0, round = 0;
        for (int i = 0; i < local && !abortFlag; ++i) {
            int n, y, x0;
            tileOf(i, n, y, x0);
            if (round > 0 && !mbarWaitRow(smemAddr(&slabEmpty[b]), static_cast<uint32_t>((round - 1) & 1), &abortFlag)) {
                abortFlag = 1;
                break;
            }
            const uint32_t slab = sSlab + b * slabBytes;
            const uint32_t full = smemAddr(&slabFull[b]);
            if (pt == 0) {
                mbarArriveExpectTx(full, txBytes);
                for (int j = cpJ; j < K16; ++j) {
                    if (j < J1) tmaLoadBox(slab + j * JS, &mapX1, pass.c1lo + 16 * j, x0 - 1, y - 1, n, full);
                    else tmaLoadBox(slab + j * JS, &mapX2, pass.c2lo + 16 * (j - J1), x0 - 1, y - 1, n, full);
                }
            }
            if (Up) {
                // the next tile's staging goes into the buffer tile i - 1 used, once all producers released it
                if (pt == 0 && i + 1 < local) {
                    if (i >= 1 && !mbarWaitRow(smemAddr(&stgEmpty[(i + 1) & 1]), static_cast<uint32_t>(((i - 1) >> 1) & 1), &abortFlag)) {
                        abortFlag = 1;
                        break;
                    }
                    issueStage(i + 1);
                }
                if (!mbarWaitRow(smemAddr(&stgFull[i & 1]), static_cast<uint32_t>((i >> 1) & 1), &abortFlag)) {
                    abortFlag = 1;
                    break;
                }
                // slab pixel r of input row d is source pixel ((x0 - 1 + r) >> 1) of source row ((y - 1 + d) >> 1);
                // the staging box starts at source pixel (x0 - 1) >> 1 and source row (y - 1) >> 1
                const int sx0 = (x0 - 1) >> 1, sy0 = (y - 1) >> 1;
                const uint32_t stg = sStg + (i & 1) * stgBytes;
                int j = 0, r = pt >> 1, d = 0, srow = 0;
                for (int e = pt; e < total; e += 128) {
                    const int sx = ((x0 - 1 + r) >> 1) - sx0;
                    stShared16(sw32(slab + j * JS + d * kSlabDStride + r * 32 + h * 16),
                               ldShared16(sw32(stg + j * SJS + srow * kStgDStride + sx * 32 + h * 16)));
                    r += 64;
                    if (r >= kSlabPx) {   // 64 < 130: at most one wrap per step
                        r -= kSlabPx;
                        if (++j == cpJ) {
                            j = 0;
                            ++d;
                            srow = ((y - 1 + d) >> 1) - sy0;
                        }
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;\n" ::);   // the tensor cores read what was written here
                mbarArrive(smemAddr(&stgEmpty[i & 1]));
            }
            if (Up) mbarArrive(full);
            if (++b == stages) { b = 0; ++round; }
        }
    } else if (warp == 8) {   // ---- MMA issue
        if (lane == 0) {
            const uint32_t idesc = instrDesc(Cout);
            const uint32_t lboB = Cout * 16;
            // descriptor start fields advance by (byte offset >> 4); shared addresses stay below 2^18, so the
            // 14-bit field never carries into the stride fields.  Weights of (tap t, k-step kk) start
            // (t * K16 + kk) * 2 * Cout * 16 bytes into the weight block.
            const uint64_t bDesc0 = smemDesc(sW, lboB, 128);
            const uint32_t bStep = 2 * Cout;
            int issued = 0, b = 0, round = 0, a = 0, aRound = 0, lastA = 0, lastRound = 0;
            for (int i = 0; i < local && !abortFlag; ++i) {
                if (!mbarWaitRow(smemAddr(&slabFull[b]), static_cast<uint32_t>(round & 1), &abortFlag) ||
                    (aRound > 0 && !mbarWaitRow(smemAddr(&accEmpty[a]), static_cast<uint32_t>((aRound - 1) & 1), &abortFlag))) {
                    abortFlag = 1;
                    break;
                }
                asm volatile("fence.proxy.async.shared::cta;\n" ::);
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                issueRowTile<K16, R>(tmem + static_cast<uint32_t>(a * R * Cout), Cout, smemDescSw32(sSlab + b * slabBytes),
                                     bDesc0, bStep, idesc);
                ummaCommit(smemAddr(&slabEmpty[b]));
                ummaCommit(smemAddr(&accFull[a]));
                issued = 1;
                lastA = a;
                lastRound = aRound;
                if (++b == stages) { b = 0; ++round; }
                if (++a == accs) { a = 0; ++aRound; }
            }
            // whatever happened, the last MMAs must be done before the tensor memory is freed
            if (issued && !mbarWaitRow(smemAddr(&accFull[lastA]), static_cast<uint32_t>(lastRound & 1), &abortFlag)) {
                unsigned long long t0 = 0;
                for (unsigned s = 0; s < kRowSpin; ++s) {   // on abort, wait on (bounded) without the abort exit
                    uint32_t done;
                    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                                 : "=r"(done)
                                 : "r"(smemAddr(&accFull[lastA])), "r"(static_cast<uint32_t>(lastRound & 1)));
                    if (done) break;
                    if ((s & 1023u) == 1023u && waitExpired(t0)) break;
                }
            }
        }
    } else if (epilogue) {   // ---- epilogue: TMEM lanes 32 (w % 4).. = tile pixels, channels [c0, c0 + Cc)
        // the wait is made warp-uniform (__all_sync) so that no lane leaves the loop alone before the
        // warp-wide tcgen05.ld and __syncwarp
        const int grp = warp & 3, Cc = Up ? Cout : Cout >> 1, c0 = Up ? 0 : (warp >> 2) * Cc;
        // registers per thread: its channels of one output row (two-row tiles have Cout <= 64, four-row ones <= 32)
        constexpr int NV = R == 4 ? 16 : R == 2 ? (Up ? 64 : 32) : (Up ? kRowMaxCout : kRowMaxCout / 2);
        int a = 0, aRound = 0;
        for (int i = 0; i < local && !abortFlag; ++i) {
            int n, y, x0;
            tileOf(i, n, y, x0);
            if (!__all_sync(0xffffffffu, mbarWaitRow(smemAddr(&accFull[a]), static_cast<uint32_t>(aRound & 1), &abortFlag))) {
                abortFlag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            const int x = x0 + grp * 32 + lane;
            const uint32_t tbase = tmem + (static_cast<uint32_t>(grp * 32) << 16) + static_cast<uint32_t>(a * R * Cout + c0);
            uint32_t pk[R][NV / 2];   // the bf16 pairs of each output row, kept for the fused pool
#pragma unroll
            for (int orow = 0; orow < R; ++orow)
#pragma unroll
                for (int q = 0; q < NV / 2; ++q) pk[orow][q] = 0u;
#pragma unroll
            for (int orow = 0; orow < R; ++orow) {
                // this thread's Cc accumulator columns of output row y + orow in flight at once, one wait; after the
                // last row the accumulator goes back to the MMA thread before the stores
                uint32_t v[NV];
                tmemLoadWait<NV>(tbase + static_cast<uint32_t>(orow * Cout), Cc, v);
                if (orow == R - 1) {
                    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
                    __syncwarp();
                    if (lane == 0) mbarArrive(smemAddr(&accEmpty[a]));
                    if (++a == accs) { a = 0; ++aRound; }
                }
                if (x < W && y + orow < H) {
                    const size_t px = (static_cast<size_t>(n) * H + y + orow) * W + x;
                    const size_t seg = ((static_cast<size_t>(n) * H + y + orow) * tilesPerRow + x0 / kRowPx) * Cout * kRowPx +
                                       static_cast<size_t>(c0) * kRowPx + (x - x0);   // channel c0 in the partial-sum layout
                    if (pass.partIn) {   // earlier passes' FP32 sums
#pragma unroll
                        for (int q = 0; q < NV / 8; ++q) {
                            if (8 * q >= Cc) break;
#pragma unroll
                            for (int k = 0; k < 8; ++k)
                                v[8 * q + k] = __float_as_uint(__uint_as_float(v[8 * q + k]) +
                                                               pass.partIn[seg + static_cast<size_t>(8 * q + k) * kRowPx]);
                        }
                    }
                    if (pass.partOut) {
#pragma unroll
                        for (int q = 0; q < NV / 8; ++q) {
                            if (8 * q >= Cc) break;
#pragma unroll
                            for (int k = 0; k < 8; ++k)
                                pass.partOut[seg + static_cast<size_t>(8 * q + k) * kRowPx] = __uint_as_float(v[8 * q + k]);
                        }
                    } else {
                        uint4* dst = reinterpret_cast<uint4*>(Y + px * Cout + c0);
                        // 16 channels (32 bytes, one sector) per 256-bit store where the channel group is 32-byte
                        // aligned, else 8 channels per 128-bit store
                        const bool wide = (c0 & 15) == 0 && (Cc & 15) == 0;
#pragma unroll
                        for (int q = 0; q < NV / 8; q += 2) {   // 8-channel units q and q + 1
                            if (8 * q >= Cc) break;
                            const bool second = 8 * (q + 1) < Cc;
                            uint32_t w8[8];
#pragma unroll
                            for (int k = 0; k < 8; ++k) {
                                const int ch = 8 * q + 2 * k;   // units q (k < 4) and q + 1 (k >= 4)
                                if (k >= 4 && !second) { w8[k] = 0u; continue; }
                                float pv = __uint_as_float(v[ch]) + sBias[c0 + ch];
                                float rv = __uint_as_float(v[ch + 1]) + sBias[c0 + ch + 1];
                                if (Relu) { pv = fmaxf(pv, 0.0f); rv = fmaxf(rv, 0.0f); }
                                const __nv_bfloat162 h = __floats2bfloat162_rn(pv, rv);
                                w8[k] = *reinterpret_cast<const uint32_t*>(&h);
                            }
                            if (wide) {
                                asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n" ::"l"(dst + q), "r"(w8[0]),
                                             "r"(w8[1]), "r"(w8[2]), "r"(w8[3]), "r"(w8[4]), "r"(w8[5]), "r"(w8[6]), "r"(w8[7])
                                             : "memory");
                            } else {
                                dst[q] = make_uint4(w8[0], w8[1], w8[2], w8[3]);
                                if (second) dst[q + 1] = make_uint4(w8[4], w8[5], w8[6], w8[7]);
                            }
                            if (R >= 2) {
#pragma unroll
                                for (int k = 0; k < 8; ++k)
                                    if (4 * q + k < NV / 2) pk[orow][4 * q + k] = w8[k];
                            }
                        }
                    }
                }
            }
            if (R >= 2 && pass.pool) {   // fused 2x2 average pool: pairs of lanes hold x and x + 1 (warp-uniform)
#pragma unroll
              for (int pr = 0; pr < R / 2; ++pr) {   // output rows y + 2 pr, y + 2 pr + 1 -> pooled row y / 2 + pr
                const bool writer = (lane & 1) == 0 && x < W && y + 2 * pr < H;
                bf16* pdst =
                    pass.pool + ((static_cast<size_t>(n) * (H >> 1) + (y >> 1) + pr) * (W >> 1) + (x >> 1)) * Cout + c0;
#pragma unroll
                for (int q = 0; q < NV / 8; ++q) {
                    if (8 * q >= Cc) break;
                    uint32_t o4[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint32_t a0 = pk[2 * pr][4 * q + k], e0 = pk[2 * pr + 1][4 * q + k];
                        const uint32_t b0 = __shfl_xor_sync(0xffffffffu, a0, 1), d0 = __shfl_xor_sync(0xffffffffu, e0, 1);
                        const float2 fa = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&a0));
                        const float2 fb = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&b0));
                        const float2 fc = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&e0));
                        const float2 fd = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&d0));
                        float s0 = 0.0f, s1 = 0.0f;
                        s0 += fa.x; s1 += fa.y;
                        s0 += fb.x; s1 += fb.y;
                        s0 += fc.x; s1 += fc.y;
                        s0 += fd.x; s1 += fd.y;
                        const __nv_bfloat162 h = __floats2bfloat162_rn(0.25f * s0, 0.25f * s1);
                        o4[k] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    if (writer) reinterpret_cast<uint4*>(pdst)[q] = make_uint4(o4[0], o4[1], o4[2], o4[3]);
                }
              }
            }
        }
    }
    __syncthreads();
    if (abortFlag && tid == 0 && errorFlag) atomicOr(errorFlag, 1u);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmemCols));
}

}  // namespace

constexpr int kTcSmem = kTcStages * (kStageABytes + kStageBBytes);

namespace {

// ---------------------------------------------------------------- weight gradient on tcgen05
// NHWC [P][C] -> kOut channel-major copies [kOut][C][P].  With kOut = 1 the plain transpose; with kOut = 3 the three
// column-shifted copies s = 0, 1, 2 (dx = s - 1: pixel (n, y, x) holds the value of (n, y, x + dx), zero where
// x + dx leaves the row), all made from one read of the input.  A block moves 64 pixels x 32 channels: 16-byte
// loads of 8 channels of one pixel (plus one halo pixel each side for the shifts) into a padded shared tile, then
// 16-byte stores of 8 pixels of one channel, a warp writing four whole 128-byte channel lines.  Needs C % 8 == 0,
// W % 8 == 0 (a stored chunk's 8 pixels share one image row) and P % 8 == 0, P < 2^31.
template <int kOut>
__global__ void __launch_bounds__(256) kPlanar(const bf16* __restrict__ in, int C, int P, int W, bf16* __restrict__ out)
{
    constexpr int kTP = 64, kTC = 32, kHalo = kOut == 3 ? 1 : 0, kRows = kTP + 2 * kHalo;
    constexpr int kStride = kTC / 2 + 1;   // 32-bit words per tile row: 16 words of channels plus one of padding
    __shared__ uint32_t tile[kRows * kStride];
    const int pb = static_cast<int>(blockIdx.x) * kTP, cb = static_cast<int>(blockIdx.y) * kTC;
    const int t = static_cast<int>(threadIdx.x);
    for (int e = t; e < kRows * 4; e += 256) {   // tile row r = pixel pb - kHalo + r, chunk q = channels cb + 8q..
        const int r = e >> 2, q = e & 3, p = pb - kHalo + r, c = cb + 8 * q;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (p >= 0 && p < P && c < C) v = *reinterpret_cast<const uint4*>(in + static_cast<size_t>(p) * C + c);
        uint32_t* dst = tile + r * kStride + 4 * q;
        dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; dst[3] = v.w;
    }
    __syncthreads();
    const unsigned short* tb = reinterpret_cast<const unsigned short*>(tile);
    for (int u = t; u < kOut * kTC * 8; u += 256) {   // unit: copy s, channel cl, 8-pixel chunk j
        const int j = u & 7, cl = (u >> 3) & (kTC - 1), s = u >> 8;
        const int c = cb + cl, p0 = pb + 8 * j;
        if (c >= C || p0 >= P) continue;
        const int dx = s - kHalo, x0 = p0 % W;
        uint32_t w[4];
        for (int k = 0; k < 4; ++k) {
            const int xa = x0 + 2 * k + dx, ra = 8 * j + 2 * k + dx + kHalo;   // source column, tile row
            const uint32_t lo = xa >= 0 && xa < W ? tb[ra * (2 * kStride) + cl] : 0u;
            const uint32_t hi = xa + 1 >= 0 && xa + 1 < W ? tb[(ra + 1) * (2 * kStride) + cl] : 0u;
            w[k] = lo | (hi << 16);
        }
        *reinterpret_cast<uint4*>(out + (static_cast<size_t>(s) * C + c) * P + p0) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// dW[tap][co][ci] += sum over pixels p of X[p shifted by the tap][ci] * dY[p][co], as one GEMM over all nine taps:
// M = the taps' input channels (row r = tap * Cin + ci, 128-row tiles, rows beyond 9 * Cin zero), N = the output
// channels (Cout, a multiple of 16) and K = the pixels.  A layer of few input channels thus fills the 128 rows with
// several taps instead of padding its output channels to 128: for 16-32 input channels 3-4.5 times fewer MMAs
// than one M = Cout GEMM per tap.  Both operands come from the channel-major copies made beforehand (dYt[co][p]
// and, per column shift dx, Xs[dx + 1][ci][p]), so one K-major 16-byte chunk is 8 consecutive pixels of one
// channel; a row's dy shift is a whole-row offset (W % 8 == 0 keeps every chunk inside one image row, whose
// validity decides the zero fill).
//
// Pipeline: kKS-pixel stages in a kStages-deep ring filled by cp.async; the stage copied kLag iterations earlier is
// handed to one thread, which issues kKS / 16 M128 x N x K16 MMAs into one TMEM accumulator and commits them to the
// stage's barrier.  The buffer refilled at iteration it last held stage it - kStages, whose MMAs were issued at
// iteration it - kStages + kLag: with kStages > kLag + 1 they had a whole iteration or more to finish, so the
// threads seldom wait on them.  Each thread keeps its rows' source offsets, dy and shared-memory offsets in
// registers and follows its chunk's image row by counting, so a stage costs its copies and little else.  Every
// wait is bounded.  The epilogue adds the CTA's partial sums into dW with FP32 atomics (neighbouring lanes hold
// neighbouring input channels of one tap: neighbouring addresses).  Grid: (row tiles, 1, pixel splits of a
// multiple of kKS pixels).
template <int kStages, int kLag, int kKS, bool kSplitFill>
__global__ void __launch_bounds__(128, 1) kWgradTc(const bf16* __restrict__ dYt, const bf16* __restrict__ Xs, int H,
                                                   int W, long long P, int Cin, int Cout, long long pixPerSplit,
                                                   float* __restrict__ dW, unsigned int* errorFlag)
{
    static_assert(kLag >= 1 && kLag < kStages && kKS % 16 == 0 && kKS >= 16 && kKS <= 64, "pipeline shape");
    constexpr int kChunks = kKS / 8;               // 16-byte chunks (8 pixels) per row and stage
    constexpr int kRowStep = 128 / kChunks;        // threads per chunk column
    constexpr int kRowsPerThread = kTcM / kRowStep;
    constexpr uint32_t kLboA = (kTcM / 8) * 128;   // distance between K-neighbouring core matrices of A
    constexpr int kStageA = kTcM * kKS * 2;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t mbar[kStages];
    __shared__ uint32_t tmemBase;
    __shared__ volatile int abortFlag;
    __shared__ volatile int lastCommit;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row0 = static_cast<int>(blockIdx.x) * kTcM;
    const int rows = 9 * Cin - row0 < kTcM ? 9 * Cin - row0 : kTcM;   // live rows of this tile
    const long long p0 = static_cast<long long>(blockIdx.z) * pixPerSplit;
    const long long p1 = p0 + pixPerSplit < P ? p0 + pixPerSplit : P;
    const int iters = p1 > p0 ? static_cast<int>((p1 - p0 + kKS - 1) / kKS) : 0;
    const int stageB = Cout * kKS * 2;
    const uint32_t sA = smemAddr(smem), sB = sA + kStages * kStageA;
    const uint32_t tmemCols = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : (Cout <= 128 ? 128 : 256));

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemAddr(&tmemBase)),
                     "r"(tmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int st = 0; st < kStages; ++st) mbarInit(smemAddr(&mbar[st]), 1);
        abortFlag = 0;
        lastCommit = -1;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    const uint32_t lboB = static_cast<uint32_t>(Cout / 8) * 128;
    const uint32_t idesc = instrDesc(Cout);
    // rows beyond the nine taps stay zero: written once here for every stage, never copied
    for (int st = 0; st < kStages; ++st)
        for (int e = tid; e < (kTcM - rows) * kChunks; e += 128) {
            const int r = rows + e / kChunks, j = e % kChunks;
            *reinterpret_cast<uint4*>(smem + st * kStageA + j * kLboA + (r >> 3) * 128 + (r & 7) * 16) =
                make_uint4(0u, 0u, 0u, 0u);
        }
    // Thread t copies chunk cj = t % kChunks (8 pixels) of rows cr, cr + kRowStep, ...: neighbouring threads read
    // one channel's contiguous pixels.  Per row: its source offset in Xs (channel plane plus dy rows), its dy and
    // its offset in the stage buffer, fixed for the whole launch.
    const int cj = tid % kChunks, cr = tid / kChunks;
    long long rowSrc[kRowsPerThread];
    int rowDy[kRowsPerThread];
    uint32_t rowDst[kRowsPerThread];
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) {
        const int r = cr + k * kRowStep;
        const int R = row0 + (r < rows ? r : 0), tap = R / Cin, ci = R - tap * Cin, dy = tap / 3 - 1, dx = tap % 3 - 1;
        rowSrc[k] = (static_cast<long long>(dx + 1) * Cin + ci) * P + static_cast<long long>(dy) * W;
        rowDy[k] = r < rows ? dy : 1 << 20;   // a dead row never passes the row test below
        rowDst[k] = cj * kLboA + (r >> 3) * 128 + (r & 7) * 16;
    }
    // the image row and column of this thread's first pixel, followed by counting from here on
    long long pc = p0 + 8 * cj;
    int x = static_cast<int>(pc % W);
    int y = static_cast<int>((pc / W) % H);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tmem = tmemBase;

    auto issueCopies = [&](int stage) {
        const uint32_t aBase = sA + stage * kStageA;
        const uint32_t bBase = sB + stage * stageB + cj * lboB;
        const bool inRange = pc < p1;
#pragma unroll
        for (int k = 0; k < kRowsPerThread; ++k) {   // A: the taps' shifted X, rows x pixels
            const int yy = y + rowDy[k];
            const bool ok = inRange && yy >= 0 && yy < H;
            if (rowDy[k] == (1 << 20)) continue;
            if (!kSplitFill) cpAsync16(aBase + rowDst[k], ok ? Xs + rowSrc[k] + pc : Xs, ok);
            else if (ok) cpAsync16Full(aBase + rowDst[k], Xs + rowSrc[k] + pc);
            else stSharedZero16(aBase + rowDst[k]);
        }
        const bf16* b = dYt + static_cast<size_t>(cr) * P + pc;
        for (int co = cr; co < Cout; co += kRowStep, b += static_cast<size_t>(kRowStep) * P) {   // B: dY^T
            const uint32_t d = bBase + (co >> 3) * 128 + (co & 7) * 16;
            if (!kSplitFill) cpAsync16(d, inRange ? b : dYt, inRange);
            else if (inRange) cpAsync16Full(d, b);
            else stSharedZero16(d);
        }
    };

    // all threads run the same barriers; a timed-out wait only raises the abort flag (no further copy or MMA)
    int fillStage = 0, mmaStage = 0;
    for (int it = 0; it < iters + kLag; ++it) {
        if (it < iters && !abortFlag) {
            bool free = true;
            if (it >= kStages) {
                const int prev = it - kStages;
                free = mbarWait(smemAddr(&mbar[fillStage]), static_cast<uint32_t>((prev / kStages) & 1));
            }
            if (free) issueCopies(fillStage);
            else abortFlag = 1;
        }
        cpAsyncCommit();
        if (it < iters) {   // the next stage's pixels: kKS columns on, into later image rows as they run out
            pc += kKS;
            x += kKS;
            while (x >= W) {
                x -= W;
                if (++y == H) y = 0;
            }
            if (++fillStage == kStages) fillStage = 0;
        }
        const int j = it - kLag;
        if (j >= 0 && j < iters) {
            cpAsyncWait<kLag>();
            asm volatile("fence.proxy.async.shared::cta;\n" ::);
            __syncthreads();
            if (tid == 0 && !abortFlag) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
#pragma unroll
                for (int k = 0; k < kKS / 16; ++k) {
                    const uint64_t da = smemDesc(sA + mmaStage * kStageA + 2 * k * kLboA, kLboA, 128);
                    const uint64_t db = smemDesc(sB + mmaStage * stageB + 2 * k * lboB, lboB, 128);
                    umma(tmem, da, db, idesc, (j > 0 || k > 0) ? 1u : 0u);
                }
                ummaCommit(smemAddr(&mbar[mmaStage]));
                lastCommit = j;
            }
            if (++mmaStage == kStages) mmaStage = 0;
        }
    }
    cpAsyncWait<0>();
    __syncthreads();
    const int last = lastCommit;
    if (last >= 0 && !mbarWait(smemAddr(&mbar[last % kStages]), static_cast<uint32_t>((last / kStages) & 1)))
        abortFlag = 1;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    __syncthreads();
    if (iters == 0) {
        // an empty split adds nothing
    } else if (abortFlag || last != iters - 1) {
        if (tid == 0 && errorFlag) atomicOr(errorFlag, 1u);
    } else {
        // warp w owns TMEM lanes 32w..32w+31 = rows (tap, ci); columns = output channels
        const int r = warp * 32 + (tid & 31), R = row0 + r;
        const int tap = R / Cin, ci = R - tap * Cin;
        float* dst = dW + static_cast<size_t>(tap) * Cout * Cin + ci;
        for (int c = 0; c < Cout; c += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                         "tcgen05.wait::ld.sync.aligned;\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr));
            if (r < rows)
                for (int k = 0; k < 16; ++k) atomicAdd(dst + static_cast<size_t>(c + k) * Cin, __uint_as_float(v[k]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmemCols));
}

}  // namespace

bool convWgradTcSupported(int N, int H, int W, int Cin, int Cout)
{
    const long long P = static_cast<long long>(N) * H * W;
    return W % 8 == 0 && P % 64 == 0 && P > 0 && P < (1LL << 31) && Cin >= 1 && Cin % 8 == 0 && Cout >= 16 &&
           Cout % 16 == 0 && Cout <= 128;
}

size_t convWgradTcScratchBytes(int N, int H, int W, int Cin, int Cout)
{
    return static_cast<size_t>(N) * H * W * (static_cast<size_t>(Cout) + 3 * static_cast<size_t>(Cin)) * sizeof(bf16);
}

namespace {

// one launch of kWgradTc<kStages, kLag, kKS>: shared memory for this launch's output channels only (kStages stages of
// the 128-row A and the Cout-row B), as many CTAs per SM as shared memory and TMEM columns (512 per SM) allow, so
// they hide one another's copy and issue latency; one wave of CTAs over the row tiles, each split at least 512
// pixels and a multiple of kKS
template <int kStages, int kLag, int kKS, bool kSplitFill>
void launchWgradTc(const bf16* dYt, const bf16* Xs, int H, int W, long long P, int Cin, int Cout, float* dW,
                   unsigned int* errorFlag, cudaStream_t st)
{
    static bool attrSet = false;
    if (!attrSet) {
        cudaFuncSetAttribute(kWgradTc<kStages, kLag, kKS, kSplitFill>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kStages * (kTcM + 128) * kKS * 2);
        attrSet = true;
    }
    const int tiles = (9 * Cin + kTcM - 1) / kTcM;
    const int smemBytes = kStages * (kTcM + Cout) * kKS * 2;
    const int tmemCols = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : 128);
    int perSm = (227 * 1024) / (smemBytes + 3 * 1024);   // plus its static shared memory and the reserve
    if (perSm > 512 / tmemCols) perSm = 512 / tmemCols;
    const int resident = perSm < 1 ? 1 : perSm;
    long long splits = (static_cast<long long>(resident) * 148 + tiles - 1) / tiles;
    long long per = (P + splits - 1) / splits;
    if (per < 512) per = 512;
    per = (per + kKS - 1) / kKS * kKS;
    splits = (P + per - 1) / per;
    kWgradTc<kStages, kLag, kKS, kSplitFill><<<dim3(static_cast<unsigned>(tiles), 1, static_cast<unsigned>(splits)), 128, smemBytes,
                                   st>>>(dYt, Xs, H, W, P, Cin, Cout, per, dW, errorFlag);
}

}  // namespace

void convWgradTc(const void* X, const void* dY, int N, int H, int W, int Cin, int Cout, float* dW, void* scratch,
                 unsigned int* errorFlag, cudaStream_t st, int variant)
{
    const long long P = static_cast<long long>(N) * H * W;
    bf16* dYt = static_cast<bf16*>(scratch);
    bf16* Xs = dYt + static_cast<size_t>(Cout) * P;
    const unsigned pt = static_cast<unsigned>((P + 63) / 64);
    kPlanar<1><<<dim3(pt, static_cast<unsigned>((Cout + 31) / 32)), 256, 0, st>>>(static_cast<const bf16*>(dY), Cout,
                                                                                  static_cast<int>(P), W, dYt);
    kPlanar<3><<<dim3(pt, static_cast<unsigned>((Cin + 31) / 32)), 256, 0, st>>>(static_cast<const bf16*>(X), Cin,
                                                                                 static_cast<int>(P), W, Xs);
    // pipeline shapes (stages, copy lag, pixels per stage)
    switch (variant == 0 ? kWgradTcDefaultVariant : variant) {
    case 1: launchWgradTc<3, 2, 64, false>(dYt, Xs, H, W, P, Cin, Cout, dW, errorFlag, st); break;
    case 2: launchWgradTc<4, 2, 64, false>(dYt, Xs, H, W, P, Cin, Cout, dW, errorFlag, st); break;
    case 3: launchWgradTc<6, 4, 32, false>(dYt, Xs, H, W, P, Cin, Cout, dW, errorFlag, st); break;
    case 4: launchWgradTc<5, 3, 32, false>(dYt, Xs, H, W, P, Cin, Cout, dW, errorFlag, st); break;
    case 5: launchWgradTc<3, 2, 64, true>(dYt, Xs, H, W, P, Cin, Cout, dW, errorFlag, st); break;
    default: launchWgradTc<5, 3, 32, true>(dYt, Xs, H, W, P, Cin, Cout, dW, errorFlag, st); break;
    }
}

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

namespace {

// shared memory: the weights, then the slab ring, then (upsampled X1) two staging buffers; R output rows per tile
long long rowFixedBytes(int C1, int C2, bool up, int Cout, int R)
{
    return ((9LL * Cout * (C1 + C2) * 2 + 1023) & ~1023LL) + (up && C1 > 0 ? 2LL * (C1 / 16) * stgJStride(R) : 0);
}

// slab buffers that fit beside the rest (at most kRowMaxStages; fewer than 2 = does not fit)
int rowStages(int C1, int C2, bool up, int Cout, int R)
{
    const long long fit =
        (kRowSmemBudget - rowFixedBytes(C1, C2, up, Cout, R)) / (static_cast<long long>((C1 + C2) / 16) * slabJStride(R));
    return static_cast<int>(fit < kRowMaxStages ? fit : kRowMaxStages);
}

int rowSmem(int C1, int C2, bool up, int Cout, int R)
{
    return static_cast<int>(rowFixedBytes(C1, C2, up, Cout, R) +
                            static_cast<long long>(rowStages(C1, C2, up, Cout, R)) * ((C1 + C2) / 16) * slabJStride(R));
}

bool rowPassFits(int n1, int n2, bool up, int Cout, int R = 1)
{
    const int cin = n1 + n2;
    if (R == 4 && (up || cin > 32 || Cout > 32)) return false;   // four-row tiles: small layers only
    return cin >= 16 && n1 % 16 == 0 && n2 % 16 == 0 && cin <= (R == 1 ? 16 * kRowMaxK16 : 64) && R * Cout <= kRowMaxCout &&
           rowStages(n1, n2, up, Cout, R) >= 2;
}

struct PassPlan {
    int c1lo, n1, c2lo, n2;
};

// Split the layer's input channels (X1's, then X2's) into passes whose weights and slabs fit in shared
// memory: one pass when the whole layer fits, else greedy runs of 16 channels.  False if no split works.
bool planRowPasses(int C1, int C2, bool up, int Cout, std::vector<PassPlan>* plan)
{
    if (!(Cout == 16 || Cout == 32 || Cout == 48 || Cout == 64 || Cout == 96 || Cout == 128) || C1 < 0 || C2 < 0 || C1 % 16 ||
        C2 % 16)
        return false;
    std::vector<PassPlan> out;
    if (rowPassFits(C1, C2, up, Cout)) {
        out.push_back({0, C1, 0, C2});
    } else {
        PassPlan cur{0, 0, 0, 0};
        for (int u = 0; u < (C1 + C2) / 16; ++u) {
            PassPlan next = cur;
            if (16 * u < C1) next.n1 += 16;
            else next.n2 += 16;
            if (rowPassFits(next.n1, next.n2, up, Cout)) {
                cur = next;
                continue;
            }
            if (cur.n1 + cur.n2 == 0) return false;   // not even 16 channels fit
            out.push_back(cur);
            cur = 16 * u < C1 ? PassPlan{16 * u, 16, 0, 0} : PassPlan{C1, 0, 16 * u - C1, 16};
            if (!rowPassFits(cur.n1, cur.n2, up, Cout)) return false;
        }
        out.push_back(cur);
    }
    if (plan) *plan = out;
    return true;
}

}  // namespace

bool convTcRowSupported(int C1, int C2, bool up, int Cout) { return planRowPasses(C1, C2, up, Cout, nullptr); }

size_t convTcRowScratchBytes(int C1, int C2, bool up, int Cout, int N, int H, int W)
{
    std::vector<PassPlan> plan;
    if (!planRowPasses(C1, C2, up, Cout, &plan) || plan.size() < 2) return 0;
    return static_cast<size_t>(N) * H * ((W + kRowPx - 1) / kRowPx) * kRowPx * Cout * sizeof(float);
}

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library links the runtime only)
PFN_cuTensorMapEncodeTiled_v12000 tensorMapEncoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            throw std::runtime_error("conv3x3TcRow: cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// NHWC bf16 tensor [N][H][W][C] read in boxes of 16 channels (32-byte rows, 32-byte swizzle) x boxW pixels x boxH
// rows, zeros outside
CUtensorMap slabMap(const void* base, int C, int N, int H, int W, int boxW, int boxH)
{
    CUtensorMap m;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(C), static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
                                static_cast<cuuint64_t>(N)};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(C) * 2, static_cast<cuuint64_t>(W) * C * 2,
                                   static_cast<cuuint64_t>(H) * W * C * 2};
    const cuuint32_t box[4] = {16, static_cast<cuuint32_t>(boxW), static_cast<cuuint32_t>(boxH), 1}, elem[4] = {1, 1, 1, 1};
    const CUresult r = tensorMapEncoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box,
                                          elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("conv3x3TcRow: cuTensorMapEncodeTiled failed");
    return m;
}

}  // namespace

bool conv3x3TcRow(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
                  const float* bias, int Cout, bool relu, void* Y, void* scratch, void* pool, unsigned int* errorFlag,
                  cudaStream_t st)
{
    bool pooled = false;
    std::vector<PassPlan> plan;
    if (!planRowPasses(C1, C2, up, Cout, &plan)) throw std::runtime_error("conv3x3TcRow: unsupported layer shape");
    if (plan.size() > 1 && (!scratch || (reinterpret_cast<uintptr_t>(scratch) & 15)))
        throw std::runtime_error("conv3x3TcRow: this layer runs in passes and needs a 16-byte aligned scratch buffer");
    if (up && ((H | W) & 1)) throw std::runtime_error("conv3x3TcRow: an upsampled input needs even H and W");
    if (static_cast<long long>(N) * H * ((W + kRowPx - 1) / kRowPx) >= (1LL << 31))
        throw std::runtime_error("conv3x3TcRow: more than 2^31 row tiles");
    if ((reinterpret_cast<uintptr_t>(X1) | reinterpret_cast<uintptr_t>(X2)) & 15)
        throw std::runtime_error("conv3x3TcRow: inputs must be 16-byte aligned");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (size_t k = 0; k < plan.size(); ++k) {
        const PassPlan& pp = plan[k];
        const bool passUp = up && pp.n1 > 0;
        // two output rows per tile (the slab's 4 input rows serve 2 outputs instead of 3 serving 1) where it fits
        // (up to 64 input channels: beyond that the unrolled descriptors of two rows spill)
        const int R = rowPassFits(pp.n1, pp.n2, passUp, Cout, 4) ? 4 : rowPassFits(pp.n1, pp.n2, passUp, Cout, 2) ? 2 : 1;
        const int smemBytes = rowSmem(pp.n1, pp.n2, passUp, Cout, R), stages = rowStages(pp.n1, pp.n2, passUp, Cout, R);
        const long long tiles = static_cast<long long>(N) * ((H + R - 1) / R) * ((W + kRowPx - 1) / kRowPx);
        CUtensorMap m1, m2;
        std::memset(&m1, 0, sizeof(m1));
        std::memset(&m2, 0, sizeof(m2));
        if (pp.n1 > 0) m1 = up ? slabMap(X1, C1, N, H / 2, W / 2, kStgPx, R + 1) : slabMap(X1, C1, N, H, W, kSlabPx, R + 2);
        if (pp.n2 > 0) m2 = slabMap(X2, C2, N, H, W, kSlabPx, R + 2);
        const bool last = k + 1 == plan.size();
        const bool poolHere = pool && last && R >= 2 && ((H | W) & 1) == 0;
        RowPass pass{pp.c1lo, pp.c2lo, C1 + C2, pp.n1 > 0 ? pp.c1lo : C1 + pp.c2lo,
                     k > 0 ? static_cast<const float*>(scratch) : nullptr, last ? nullptr : static_cast<float*>(scratch),
                     poolHere ? static_cast<bf16*>(pool) : nullptr};
        pooled = pooled || poolHere;
        auto launch = [&](auto kernel) {
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smemBytes);
            int per = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kRowThreads, smemBytes) != cudaSuccess || per < 1) per = 1;
            // accumulator ring: up to kRowMaxAccs tiles of R x Cout columns in a power-of-two allocation, every
            // resident CTA holding its tensor memory at once (512 columns per SM)
            int tmemCols = 32;
            while (tmemCols < 2 * R * Cout) tmemCols *= 2;
            if (per * tmemCols > 512) per = 512 / tmemCols;
            while (tmemCols / (R * Cout) < kRowMaxAccs && per * tmemCols * 2 <= 512) tmemCols *= 2;
            const int accs = tmemCols / (R * Cout) < kRowMaxAccs ? tmemCols / (R * Cout) : kRowMaxAccs;
            const long long grid = tiles < static_cast<long long>(sms) * per ? tiles : static_cast<long long>(sms) * per;
            // launched as a programmatic dependent of the previous kernel in the stream (the kernel waits
            // with griddepcontrol.wait before it touches activations)
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(static_cast<unsigned>(grid));
            cfg.blockDim = dim3(kRowThreads);
            cfg.dynamicSmemBytes = static_cast<size_t>(smemBytes);
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, m1, m2, pp.n1, pp.n2, N, H, W, static_cast<const bf16*>(Wk),
                                                     bias, Cout, static_cast<bf16*>(Y), pass, stages, accs, tmemCols, errorFlag);
            if (e != cudaSuccess) throw std::runtime_error(std::string("conv3x3TcRow: launch failed: ") + cudaGetErrorString(e));
        };
        auto byK = [&](auto relu_, auto up_, auto r_) {
            constexpr bool RL = decltype(relu_)::value, U = decltype(up_)::value;
            constexpr int RR = decltype(r_)::value;
            switch ((pp.n1 + pp.n2) / 16) {
                case 1: launch(kConvTcRow<RL, U, 1, RR>); break;
                case 2: launch(kConvTcRow<RL, U, 2, RR>); break;
                case 3:
                    if constexpr (RR <= 2) launch(kConvTcRow<RL, U, 3, RR>);
                    break;
                case 4:
                    if constexpr (RR <= 2) launch(kConvTcRow<RL, U, 4, RR>);
                    break;
                case 5:
                    if constexpr (RR == 1) launch(kConvTcRow<RL, U, 5, 1>);
                    break;
                case 6:
                    if constexpr (RR == 1) launch(kConvTcRow<RL, U, 6, 1>);
                    break;
                default: throw std::runtime_error("conv3x3TcRow: a pass takes 16 to 96 channels");
            }
        };
        auto byR = [&](auto relu_, auto up_) {
            if (R == 4) byK(relu_, up_, std::integral_constant<int, 4>{});
            else if (R == 2) byK(relu_, up_, std::integral_constant<int, 2>{});
            else byK(relu_, up_, std::integral_constant<int, 1>{});
        };
        using T = std::true_type;
        using F = std::false_type;
        if (relu) {
            if (passUp) byR(T{}, T{});
            else byR(T{}, F{});
        } else {
            if (passUp) byR(F{}, T{});
            else byR(F{}, F{});
        }
    }
    return pooled;
}

void waitTimeoutProbe(unsigned int* dStatus, unsigned long long* dNs, cudaStream_t st)
{
    kWaitTimeoutProbe<<<1, 32, 0, st>>>(dStatus, dNs);
}

}  // namespace dn
}  // namespace bte
