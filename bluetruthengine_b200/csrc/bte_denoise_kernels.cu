// bte_denoise_kernels.cu -- kernels of the learned denoiser (replaces the
// reference's vendor denoiser stage, src/host/denoiser.cu:72-109).
//
// Tensors are NHWC bf16 with channel counts that are multiples of 16.  The
// 3x3 convolutions run on the tensor cores as implicit GEMMs with BF16
// operands and FP32 accumulation (mma.sync m16n8k16):
//   forward / data gradient:  Y[p][co] = act(b[co] + sum_{tap,ci} X[p+off(tap)][ci] * Wk[tap][co][ci])
//     (the data gradient is the same product with the taps mirrored and the
//      channel roles swapped, Wd[tap][ci][co] = Wk[8-tap][co][ci])
//   weight gradient:          dW[tap][co][ci] += sum_p dY[p][co] * X[p+off(tap)][ci]
//     (pixels are the reduction axis; both operands are pixel-major in
//      memory, so tiles go through shared memory and ldmatrix.trans)
// plus pooling, upsample+concatenate, feature assembly, loss and Adam.
#include "bte_denoise.h"

#include <cuda_bf16.h>

#include <cstdint>

namespace bte {
namespace dn {

namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t ld32(const bf16* p) { return __ldg(reinterpret_cast<const unsigned int*>(p)); }

__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm4t(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p)
{
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
}

__device__ __forceinline__ uint32_t packBf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// ------------------------------------------------------------ 3x3 convolution (forward / data gradient)
// The input is concat(Up ? nearest-upsample-2x(X1) : X1, X2): C1 channels
// from X1 ([N, H/2, W/2, C1] when Up, else [N, H, W, C1]) followed by C2
// channels of X2 ([N, H, W, C2]; C2 may be 0), so the decoder's
// upsample-and-concatenate is read in place.  A CTA computes 16 consecutive
// pixels of one row x 8*NT output channels; its four warps split the nine
// taps (w, w+4, w+8) and their partial sums meet in shared memory, so that
// the small low-resolution layers still put enough warps on the machine.
// Per 16-channel step a warp issues one m16n8k16 BF16 MMA per 8 output
// channels; A fragments are gathered from global memory (the neighbourhood
// re-reads hit L1), B fragments from the weights, one step ahead.
template <int NT>
struct ConvFrag {
    uint32_t a[4];
    uint32_t b[NT][2];
};

template <int NT, bool Up>
__device__ __forceinline__ void convLoad(ConvFrag<NT>& f, const bf16* __restrict__ X1, int C1, const bf16* __restrict__ X2,
                                         int C2, int n, int H, int W, int y, int xa, int xb, int tap, int c0,
                                         const bf16* __restrict__ Wk, int Cout, int co0, int g, int t)
{
    const int Cin = C1 + C2;
    const int yy = y + tap / 3 - 1;
    const int dx = tap % 3 - 1;
    const int xxa = xa + dx, xxb = xb + dx;
    const bool rowOk = yy >= 0 && yy < H;
    const bool okA = rowOk && xxa >= 0 && xxa < W;
    const bool okB = rowOk && xxb >= 0 && xxb < W;
    const bf16 *pa, *pb;
    if (c0 < C1) {
        const int Hs = Up ? H / 2 : H, Ws = Up ? W / 2 : W;
        const int ys = rowOk ? (Up ? yy / 2 : yy) : 0;
        const size_t rowBase = (static_cast<size_t>(n) * Hs + ys) * Ws;
        pa = X1 + (rowBase + (okA ? (Up ? xxa / 2 : xxa) : 0)) * C1 + c0 + 2 * t;
        pb = X1 + (rowBase + (okB ? (Up ? xxb / 2 : xxb) : 0)) * C1 + c0 + 2 * t;
    } else {
        const size_t rowBase = (static_cast<size_t>(n) * H + (rowOk ? yy : 0)) * W;
        pa = X2 + (rowBase + (okA ? xxa : 0)) * C2 + (c0 - C1) + 2 * t;
        pb = X2 + (rowBase + (okB ? xxb : 0)) * C2 + (c0 - C1) + 2 * t;
    }
    f.a[0] = okA ? ld32(pa) : 0u;
    f.a[1] = okB ? ld32(pb) : 0u;
    f.a[2] = okA ? ld32(pa + 8) : 0u;
    f.a[3] = okB ? ld32(pb + 8) : 0u;
    const bf16* wt = Wk + (static_cast<size_t>(tap) * Cout + co0 + g) * Cin + c0 + 2 * t;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        f.b[j][0] = ld32(wt + static_cast<size_t>(j * 8) * Cin);
        f.b[j][1] = ld32(wt + static_cast<size_t>(j * 8) * Cin + 8);
    }
}

template <int NT>
__device__ __forceinline__ void convMma(float (&acc)[NT][4], const ConvFrag<NT>& f)
{
#pragma unroll
    for (int j = 0; j < NT; ++j) mma16816(acc[j], f.a[0], f.a[1], f.a[2], f.a[3], f.b[j][0], f.b[j][1]);
}

template <int NT, bool Relu, bool Up, bool Split>
__global__ void __launch_bounds__(128) kConv3x3(const bf16* __restrict__ X1, int C1, const bf16* __restrict__ X2, int C2,
                                                int H, int W, const bf16* __restrict__ Wk, const float* __restrict__ bias,
                                                int Cout, int colBlocks, bf16* __restrict__ Y)
{
    __shared__ float part[Split ? 4 : 1][16][8 * NT + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int n = blockIdx.z / colBlocks;
    const int co0 = (blockIdx.z - n * colBlocks) * (8 * NT);
    const int y = blockIdx.y;
    const int x0 = Split ? blockIdx.x * 16 : blockIdx.x * 64 + warp * 16;
    if (!Split && x0 >= W) return;
    const int xa = x0 + g, xb = x0 + g + 8;
    const int Cin = C1 + C2;
    const int chunks = Cin / 16;
    const int steps = (Split ? (warp == 0 ? 3 : 2) : 9) * chunks;   // split: taps warp, warp + 4, warp + 8
    auto tapOf = [&](int step) { return Split ? warp + 4 * (step / chunks) : step / chunks; };
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    ConvFrag<NT> fa, fb;
    convLoad<NT, Up>(fa, X1, C1, X2, C2, n, H, W, y, xa, xb, tapOf(0), 0, Wk, Cout, co0, g, t);
    for (int s = 0; s < steps; s += 2) {
        if (s + 1 < steps)
            convLoad<NT, Up>(fb, X1, C1, X2, C2, n, H, W, y, xa, xb, tapOf(s + 1), 16 * ((s + 1) % chunks), Wk, Cout, co0,
                             g, t);
        convMma<NT>(acc, fa);
        if (s + 1 >= steps) break;
        if (s + 2 < steps)
            convLoad<NT, Up>(fa, X1, C1, X2, C2, n, H, W, y, xa, xb, tapOf(s + 2), 16 * ((s + 2) % chunks), Wk, Cout, co0,
                             g, t);
        convMma<NT>(acc, fb);
    }
    if (!Split) {
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int co = co0 + j * 8 + 2 * t;
            const float b0 = bias ? bias[co] : 0.0f, b1 = bias ? bias[co + 1] : 0.0f;
            float v00 = acc[j][0] + b0, v01 = acc[j][1] + b1, v10 = acc[j][2] + b0, v11 = acc[j][3] + b1;
            if (Relu) {
                v00 = fmaxf(v00, 0.0f); v01 = fmaxf(v01, 0.0f); v10 = fmaxf(v10, 0.0f); v11 = fmaxf(v11, 0.0f);
            }
            const size_t rowOut = (static_cast<size_t>(n) * H + y) * W;
            if (xa < W) *reinterpret_cast<uint32_t*>(Y + (rowOut + xa) * Cout + co) = packBf16(v00, v01);
            if (xb < W) *reinterpret_cast<uint32_t*>(Y + (rowOut + xb) * Cout + co) = packBf16(v10, v11);
        }
        return;
    }
    const int pw = Split ? warp : 0;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        part[pw][g][j * 8 + 2 * t] = acc[j][0];
        part[pw][g][j * 8 + 2 * t + 1] = acc[j][1];
        part[pw][g + 8][j * 8 + 2 * t] = acc[j][2];
        part[pw][g + 8][j * 8 + 2 * t + 1] = acc[j][3];
    }
    __syncthreads();
    // 16 pixels x 4*NT channel pairs, summed over the four warps
    for (int e = threadIdx.x; e < 16 * 4 * NT; e += 128) {
        const int px = e / (4 * NT), cp = 2 * (e % (4 * NT));
        const int x = x0 + px;
        if (x >= W) continue;
        float v0 = 0.0f, v1 = 0.0f;
#pragma unroll
        for (int q = 0; q < (Split ? 4 : 1); ++q) { v0 += part[q][px][cp]; v1 += part[q][px][cp + 1]; }
        const int co = co0 + cp;
        if (bias) { v0 += bias[co]; v1 += bias[co + 1]; }
        if (Relu) { v0 = fmaxf(v0, 0.0f); v1 = fmaxf(v1, 0.0f); }
        *reinterpret_cast<uint32_t*>(Y + ((static_cast<size_t>(n) * H + y) * W + x) * Cout + co) = packBf16(v0, v1);
    }
}

// ------------------------------------------------------------ weight gradient
// grid: x = co tiles (64) * ci tiles (64), y = tap, z = pixel splits.  Each
// CTA reduces its pixel range in chunks of 32 staged in shared memory and
// adds its 64x64 partial into dW (FP32 atomics).  Warps form a 2x2 grid of
// 32x32 sub-tiles.
constexpr int kWgPix = 32;
constexpr int kWgLd = 72;   // row pitch in elements (64 + 8 keeps ldmatrix rows on distinct banks)

__global__ void __launch_bounds__(128) kConvWgrad(const bf16* __restrict__ X, const bf16* __restrict__ dY, int N, int H,
                                                  int W, int Cin, int Cout, int pixPerSplit, float* __restrict__ dW)
{
    __shared__ __align__(16) bf16 sY[kWgPix][kWgLd];
    __shared__ __align__(16) bf16 sX[kWgPix][kWgLd];
    const int ciTiles = (Cin + 63) / 64;
    const int co0 = (blockIdx.x / ciTiles) * 64;
    const int ci0 = (blockIdx.x % ciTiles) * 64;
    const int tap = blockIdx.y;
    const int dyy = tap / 3 - 1, dxx = tap % 3 - 1;
    const long long total = static_cast<long long>(N) * H * W;
    const long long p0 = static_cast<long long>(blockIdx.z) * pixPerSplit;
    const long long p1 = p0 + pixPerSplit < total ? p0 + pixPerSplit : total;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.0f;
    for (long long pc = p0; pc < p1; pc += kWgPix) {
        // stage: 32 pixels x 64 channels of dY and of the tap-shifted X, 16-byte vectors (2 per thread each)
        for (int v = threadIdx.x; v < kWgPix * 8; v += 128) {
            const int r = v >> 3, c8 = (v & 7) * 8;
            const long long p = pc + r;
            uint4 yv = make_uint4(0u, 0u, 0u, 0u), xv = make_uint4(0u, 0u, 0u, 0u);
            if (p < p1) {
                if (co0 + c8 < Cout) yv = __ldg(reinterpret_cast<const uint4*>(dY + p * Cout + co0 + c8));
                const int x = static_cast<int>(p % W);
                const long long ny = p / W;
                const int y = static_cast<int>(ny % H);
                const int xs = x + dxx, ys = y + dyy;
                if (ci0 + c8 < Cin && xs >= 0 && xs < W && ys >= 0 && ys < H)
                    xv = __ldg(reinterpret_cast<const uint4*>(X + (p + static_cast<long long>(dyy) * W + dxx) * Cin + ci0 + c8));
            }
            *reinterpret_cast<uint4*>(&sY[r][c8]) = yv;
            *reinterpret_cast<uint4*>(&sX[r][c8]) = xv;
        }
        __syncthreads();
        const int i = lane & 7, mat = lane >> 3;
#pragma unroll
        for (int kk = 0; kk < kWgPix; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {   // A = dY^T: matrices (m+0,k+0) (m+8,k+0) (m+0,k+8) (m+8,k+8)
                const int kOff = (mat >> 1) * 8, mOff = (mat & 1) * 8;
                ldsm4t(a[mi][0], a[mi][1], a[mi][2], a[mi][3], &sY[kk + kOff + i][wm + mi * 16 + mOff]);
            }
#pragma unroll
            for (int nj = 0; nj < 4; nj += 2) {   // B = X: matrices (n+0,k+0) (n+0,k+8) (n+8,k+0) (n+8,k+8)
                const int kOff = (mat & 1) * 8, nOff = (mat >> 1) * 8;
                ldsm4t(b[nj][0], b[nj][1], b[nj + 1][0], b[nj + 1][1], &sX[kk + kOff + i][wn + nj * 8 + nOff]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int nj = 0; nj < 4; ++nj)
                    mma16816(acc[mi][nj], a[mi][0], a[mi][1], a[mi][2], a[mi][3], b[nj][0], b[nj][1]);
        }
        __syncthreads();
    }
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) {
            const int co = co0 + wm + mi * 16 + g;
            const int ci = ci0 + wn + nj * 8 + 2 * t;
            if (ci >= Cin) continue;
            float* base = dW + static_cast<size_t>(tap) * Cout * Cin;
            if (co < Cout) {
                atomicAdd(base + static_cast<size_t>(co) * Cin + ci, acc[mi][nj][0]);
                atomicAdd(base + static_cast<size_t>(co) * Cin + ci + 1, acc[mi][nj][1]);
            }
            if (co + 8 < Cout) {
                atomicAdd(base + static_cast<size_t>(co + 8) * Cin + ci, acc[mi][nj][2]);
                atomicAdd(base + static_cast<size_t>(co + 8) * Cin + ci + 1, acc[mi][nj][3]);
            }
        }
}

// bias gradient: db[c] += sum_p dY[p][c].  A block of 256 threads sums a contiguous pixel range: thread t reads
// the 16-byte chunk t % (C / 8) (8 channels) of every (256 / (C / 8))-th pixel, so a warp reads neighbouring
// pixels' whole channel rows; the threads' sums are combined per channel in shared memory and added to db with one
// atomic per channel and block.  C % 8 == 0, 8 <= C <= 256.
__global__ void __launch_bounds__(256) kBiasGrad8(const bf16* __restrict__ dY, long long total, int C,
                                                  long long pixPerCta, float* __restrict__ db)
{
    __shared__ float part[256 * 8];
    const int chunks = C >> 3, lanes = 256 / chunks, t = static_cast<int>(threadIdx.x);
    const int chunk = t % chunks, lane = t / chunks;
    const long long p0 = static_cast<long long>(blockIdx.x) * pixPerCta;
    const long long p1 = p0 + pixPerCta < total ? p0 + pixPerCta : total;
    float s[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (lane < lanes) {
#pragma unroll 4
        for (long long p = p0 + lane; p < p1; p += lanes) {
            const uint4 v = *reinterpret_cast<const uint4*>(dY + p * C + 8 * chunk);
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
            for (int k = 0; k < 4; ++k) {
                s[2 * k] += __low2float(h[k]);
                s[2 * k + 1] += __high2float(h[k]);
            }
        }
    }
    for (int k = 0; k < 8; ++k) part[t * 8 + k] = s[k];   // threads beyond lanes * chunks hold zeros
    __syncthreads();
    for (int c = t; c < C; c += 256) {
        const int ch = c >> 3, k = c & 7;
        float acc = 0.0f;
        for (int l = 0; l < lanes; ++l) acc += part[(l * chunks + ch) * 8 + k];
        atomicAdd(db + c, acc);
    }
}

// bias gradient for channel counts that are not a multiple of 8: one thread per channel pair, CTA over a pixel range
__global__ void kBiasGrad(const bf16* __restrict__ dY, long long total, int C, int pixPerCta, float* __restrict__ db)
{
    const int c2 = threadIdx.x;   // blockDim = C / 2
    const long long p0 = static_cast<long long>(blockIdx.x) * pixPerCta;
    const long long p1 = p0 + pixPerCta < total ? p0 + pixPerCta : total;
    float s0 = 0.0f, s1 = 0.0f;
    for (long long p = p0; p < p1; ++p) {
        const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(dY + p * C + 2 * c2);
        s0 += __bfloat162float(v.x);
        s1 += __bfloat162float(v.y);
    }
    atomicAdd(db + 2 * c2, s0);
    atomicAdd(db + 2 * c2 + 1, s1);
}

// dYm = dY where Y > 0 (ReLU derivative), elementwise over 16-byte groups of 8 bf16
__global__ void kReluMask8(const uint4* __restrict__ Y, const uint4* dY, uint4* out, long long n8)   // out may be dY
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n8;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const uint4 y = Y[i];
        uint4 d = dY[i];
        const uint32_t* yw = reinterpret_cast<const uint32_t*>(&y);
        uint32_t* dw = reinterpret_cast<uint32_t*>(&d);
        for (int k = 0; k < 4; ++k) {
            const __nv_bfloat162 yy = *reinterpret_cast<const __nv_bfloat162*>(&yw[k]);
            const uint32_t keepLo = __low2float(yy) > 0.0f ? 0x0000ffffu : 0u;
            const uint32_t keepHi = __high2float(yy) > 0.0f ? 0xffff0000u : 0u;
            dw[k] &= keepLo | keepHi;
        }
        out[i] = d;
    }
}

// dYm = dY where Y > 0 (ReLU derivative), elementwise over bf16 pairs
__global__ void kReluMask(const bf16* __restrict__ Y, const bf16* __restrict__ dY, bf16* __restrict__ out, long long n2)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n2;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const __nv_bfloat162 y = reinterpret_cast<const __nv_bfloat162*>(Y)[i];
        __nv_bfloat162 d = reinterpret_cast<const __nv_bfloat162*>(dY)[i];
        if (!(__bfloat162float(y.x) > 0.0f)) d.x = __float2bfloat16(0.0f);
        if (!(__bfloat162float(y.y) > 0.0f)) d.y = __float2bfloat16(0.0f);
        reinterpret_cast<__nv_bfloat162*>(out)[i] = d;
    }
}

// ------------------------------------------------------------ pooling / upsampling
// 2x2 average pool: [N, H, W, C] -> [N, H/2, W/2, C]
// The pool, upsample and output kernels are launched as programmatic dependents of the convolution before
// them (launchAfterConv): they wait for it here before touching memory.
__device__ __forceinline__ void waitForPredecessor() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

__global__ void kPool2(const bf16* __restrict__ X, int N, int H, int W, int C, bf16* __restrict__ Y)
{
    waitForPredecessor();
    const int Ho = H / 2, Wo = W / 2, C2 = C / 2;
    const long long total = static_cast<long long>(N) * Ho * Wo * C2;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i % C2);
        long long r = i / C2;
        const int x = static_cast<int>(r % Wo); r /= Wo;
        const int y = static_cast<int>(r % Ho);
        const int n = static_cast<int>(r / Ho);
        float s0 = 0.0f, s1 = 0.0f;
        for (int k = 0; k < 4; ++k) {
            const size_t src = ((static_cast<size_t>(n) * H + 2 * y + (k >> 1)) * W + 2 * x + (k & 1)) * C + 2 * c;
            const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(X + src);
            s0 += __bfloat162float(v.x);
            s1 += __bfloat162float(v.y);
        }
        reinterpret_cast<__nv_bfloat162*>(Y)[i] = __floats2bfloat162_rn(0.25f * s0, 0.25f * s1);
    }
}

// gradient of the pool, added into dX (dX += dY / 4 on each of the 4 inputs)
__global__ void kPool2Back(const bf16* __restrict__ dY, int N, int H, int W, int C, bf16* __restrict__ dX)
{
    const int C2 = C / 2;
    const long long total = static_cast<long long>(N) * H * W * C2;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i % C2);
        long long r = i / C2;
        const int x = static_cast<int>(r % W); r /= W;
        const int y = static_cast<int>(r % H);
        const int n = static_cast<int>(r / H);
        const size_t src = ((static_cast<size_t>(n) * (H / 2) + y / 2) * (W / 2) + x / 2) * C + 2 * c;
        const __nv_bfloat162 g2 = *reinterpret_cast<const __nv_bfloat162*>(dY + src);
        __nv_bfloat162& d = reinterpret_cast<__nv_bfloat162*>(dX)[i];
        d = __floats2bfloat162_rn(__bfloat162float(d.x) + 0.25f * __bfloat162float(g2.x),
                                  __bfloat162float(d.y) + 0.25f * __bfloat162float(g2.y));
    }
}

// out[N, H, W, Ca + Cb] = concat(nearest-upsample-2x(A[N, H/2, W/2, Ca]), B[N, H, W, Cb])
__global__ void kUpCat(const bf16* __restrict__ A, int Ca, const bf16* __restrict__ B, int Cb, int N, int H, int W,
                       bf16* __restrict__ out)
{
    const int C = Ca + Cb, C2 = C / 2;
    const long long total = static_cast<long long>(N) * H * W * C2;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c = 2 * static_cast<int>(i % C2);
        const long long pix = i / C2;
        const int x = static_cast<int>(pix % W);
        const long long r = pix / W;
        const int y = static_cast<int>(r % H);
        const int n = static_cast<int>(r / H);
        __nv_bfloat162 v;
        if (c < Ca) v = *reinterpret_cast<const __nv_bfloat162*>(A + ((static_cast<size_t>(n) * (H / 2) + y / 2) * (W / 2) + x / 2) * Ca + c);
        else v = *reinterpret_cast<const __nv_bfloat162*>(B + pix * Cb + (c - Ca));
        reinterpret_cast<__nv_bfloat162*>(out)[i] = v;
    }
}

// nearest 2x upsampling Y[N][2Hs][2Ws][C] = X[N][Hs][Ws][C]: one 16-byte chunk of a source pixel per
// thread, written to its four destination pixels
__global__ void kUpsample2(const uint4* __restrict__ X, int N, int Hs, int Ws, int C8, uint4* __restrict__ Y)
{
    waitForPredecessor();
    const long long total = static_cast<long long>(N) * Hs * Ws * C8;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i % C8);
        long long r = i / C8;
        const int x = static_cast<int>(r % Ws); r /= Ws;
        const int y = static_cast<int>(r % Hs);
        const int n = static_cast<int>(r / Hs);
        const uint4 v = X[i];
        const size_t row0 = (static_cast<size_t>(n) * 2 * Hs + 2 * y) * (2 * Ws), row1 = row0 + 2 * Ws;
        Y[(row0 + 2 * x) * C8 + c] = v;
        Y[(row0 + 2 * x + 1) * C8 + c] = v;
        Y[(row1 + 2 * x) * C8 + c] = v;
        Y[(row1 + 2 * x + 1) * C8 + c] = v;
    }
}

// gradient of kUpCat: dA = sum of the 2x2 block (written), dB = slice (written, or added if addB)
__global__ void kUpCatBack(const bf16* __restrict__ dOut, int Ca, int Cb, int N, int H, int W, bf16* __restrict__ dA,
                           bf16* __restrict__ dB, int addB)
{
    const int C = Ca + Cb;
    const int Ho = H / 2, Wo = W / 2;
    // part 1: dA over the low-resolution grid
    const long long totalA = static_cast<long long>(N) * Ho * Wo * (Ca / 2);
    const long long totalB = static_cast<long long>(N) * H * W * (Cb / 2);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < totalA + totalB;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if (i < totalA) {
            const int c = 2 * static_cast<int>(i % (Ca / 2));
            long long r = i / (Ca / 2);
            const int x = static_cast<int>(r % Wo); r /= Wo;
            const int y = static_cast<int>(r % Ho);
            const int n = static_cast<int>(r / Ho);
            float s0 = 0.0f, s1 = 0.0f;
            for (int k = 0; k < 4; ++k) {
                const size_t src = ((static_cast<size_t>(n) * H + 2 * y + (k >> 1)) * W + 2 * x + (k & 1)) * C + c;
                const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(dOut + src);
                s0 += __bfloat162float(v.x);
                s1 += __bfloat162float(v.y);
            }
            reinterpret_cast<__nv_bfloat162*>(dA)[i] = __floats2bfloat162_rn(s0, s1);
        } else {
            const long long j = i - totalA;
            const int c = 2 * static_cast<int>(j % (Cb / 2));
            const long long pix = j / (Cb / 2);
            const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(dOut + pix * C + Ca + c);
            __nv_bfloat162& d = reinterpret_cast<__nv_bfloat162*>(dB)[j];
            if (addB) d = __floats2bfloat162_rn(__bfloat162float(d.x) + __bfloat162float(v.x),
                                                __bfloat162float(d.y) + __bfloat162float(v.y));
            else d = v;
        }
    }
}

// ------------------------------------------------------------ features, output, loss
// Network input [N, Hp, Wp, 16] from radiance [N, H, W, 3] and features
// [N, H, W, 6] (albedo, normal), edge-replicated to the padded size:
// channels log(1 + max(L, 0)), albedo, normal, zeros.
__global__ void kAssemble(const float* __restrict__ rad, const float* __restrict__ feat, int N, int H, int W, int Hp,
                          int Wp, bf16* __restrict__ out)
{
    const long long total = static_cast<long long>(N) * Hp * Wp;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % Wp);
        const long long r = i / Wp;
        const int y = static_cast<int>(r % Hp);
        const int n = static_cast<int>(r / Hp);
        const size_t src = (static_cast<size_t>(n) * H + (y < H ? y : H - 1)) * W + (x < W ? x : W - 1);
        float v[16];
        for (int c = 0; c < 3; ++c) v[c] = log1pf(fmaxf(rad[3 * src + c], 0.0f));
        for (int c = 0; c < 6; ++c) v[3 + c] = feat ? feat[6 * src + c] : 0.0f;
        for (int c = 9; c < 16; ++c) v[c] = 0.0f;
        uint32_t w[8];
        for (int k = 0; k < 8; ++k) w[k] = packBf16(v[2 * k], v[2 * k + 1]);
        uint4* o = reinterpret_cast<uint4*>(out + i * 16);
        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// prediction (log space) = network output channels 0-2 + input log radiance
// (residual); radiance = expm1 of it, cropped to [N, H, W, 3]
__global__ void kOutput(const bf16* __restrict__ net, const bf16* __restrict__ in, int N, int H, int W, int Hp, int Wp,
                        float* __restrict__ rad)
{
    waitForPredecessor();
    const long long total = static_cast<long long>(N) * H * W;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % W);
        const long long r = i / W;
        const int y = static_cast<int>(r % H);
        const int n = static_cast<int>(r / H);
        const size_t q = (static_cast<size_t>(n) * Hp + y) * Wp + x;
        for (int c = 0; c < 3; ++c) {
            const float l = __bfloat162float(net[q * 16 + c]) + __bfloat162float(in[q * 16 + c]);
            rad[3 * i + c] = fmaxf(expm1f(l), 0.0f);
        }
    }
}

// L1 loss in log space against target radiance [N, H, W, 3]; writes the
// gradient w.r.t. the network output (16 channels, zero beyond 3) and adds
// the summed |error| into *lossSum.
__global__ void kLossL1(const bf16* __restrict__ net, const bf16* __restrict__ in, const float* __restrict__ target,
                        long long total, float scale, bf16* __restrict__ dNet, float* __restrict__ lossSum)
{
    float local = 0.0f;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        uint32_t w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        float gch[3];
        for (int c = 0; c < 3; ++c) {
            const float pred = __bfloat162float(net[i * 16 + c]) + __bfloat162float(in[i * 16 + c]);
            const float tgt = log1pf(fmaxf(target[3 * i + c], 0.0f));
            const float e = pred - tgt;
            local += fabsf(e);
            gch[c] = e > 0.0f ? scale : (e < 0.0f ? -scale : 0.0f);
        }
        w[0] = packBf16(gch[0], gch[1]);
        w[1] = packBf16(gch[2], 0.0f);
        uint4* o = reinterpret_cast<uint4*>(dNet + i * 16);
        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(lossSum, local);
}

// ------------------------------------------------------------ parameters
// Adam on FP32 master weights; refreshes the bf16 forward copy and, for
// weight tensors, the mirrored/transposed copy used by the data gradient.
__global__ void kAdam(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                      long long n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float gr = grad[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gr;
        const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// forward copy Wk[tap][co][ci] (bf16) and data-gradient copy Wd[tap][ci][co] = Wk[8-tap][co][ci]
__global__ void kWeightCopies(const float* __restrict__ w, int Cin, int Cout, bf16* __restrict__ wk, bf16* __restrict__ wd)
{
    const long long n = 9LL * Cin * Cout;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int ci = static_cast<int>(i % Cin);
        const long long r = i / Cin;
        const int co = static_cast<int>(r % Cout);
        const int tap = static_cast<int>(r / Cout);
        const bf16 b = __float2bfloat16(w[i]);
        wk[i] = b;
        if (wd) wd[(static_cast<size_t>(8 - tap) * Cin + ci) * Cout + co] = b;
    }
}

int gridFor(long long n, int block = 256)
{
    long long g = (n + block - 1) / block;
    if (g > 148LL * 32) g = 148LL * 32;
    return static_cast<int>(g < 1 ? 1 : g);
}

template <bool Relu, bool Up, bool Split>
void launchConvNT(int nt, dim3 grid, const bf16* X1, int C1, const bf16* X2, int C2, int H, int W, const bf16* Wk,
                  const float* bias, int Cout, int colBlocks, bf16* Y, cudaStream_t st)
{
#define BTE_CONV_CASE(K) \
    case K: kConv3x3<K, Relu, Up, Split><<<grid, 128, 0, st>>>(X1, C1, X2, C2, H, W, Wk, bias, Cout, colBlocks, Y); break;
    switch (nt) {
    BTE_CONV_CASE(1) BTE_CONV_CASE(2) BTE_CONV_CASE(3) BTE_CONV_CASE(4) BTE_CONV_CASE(5) BTE_CONV_CASE(6) BTE_CONV_CASE(7)
    default: kConv3x3<8, Relu, Up, Split><<<grid, 128, 0, st>>>(X1, C1, X2, C2, H, W, Wk, bias, Cout, colBlocks, Y); break;
    }
#undef BTE_CONV_CASE
}

template <bool Relu, bool Up>
void launchConv(int nt, int N, int H, int W, const bf16* X1, int C1, const bf16* X2, int C2, const bf16* Wk,
                const float* bias, int Cout, int colBlocks, bf16* Y, cudaStream_t st)
{
    // Unsplit CTAs (64 pixels, each warp all nine taps) when they fill the
    // machine several times over; otherwise 16-pixel CTAs whose warps split the taps.
    const long long whole = static_cast<long long>((W + 63) / 64) * H * N * colBlocks;
    if (whole >= 148LL * 16)
        launchConvNT<Relu, Up, false>(nt, dim3((W + 63) / 64, H, N * colBlocks), X1, C1, X2, C2, H, W, Wk, bias, Cout,
                                      colBlocks, Y, st);
    else
        launchConvNT<Relu, Up, true>(nt, dim3((W + 15) / 16, H, N * colBlocks), X1, C1, X2, C2, H, W, Wk, bias, Cout,
                                     colBlocks, Y, st);
}

}  // namespace

// largest 8*nt (nt <= 8) dividing cout
static int pickNT(int cout)
{
    for (int nt = 8; nt >= 1; --nt)
        if (cout % (8 * nt) == 0) return nt;
    return 1;
}

void conv3x3(const void* X, int N, int H, int W, int Cin, const void* Wk, const float* bias, int Cout, bool relu, void* Y,
             cudaStream_t st)
{
    conv3x3Cat(X, Cin, false, nullptr, 0, N, H, W, Wk, bias, Cout, relu, Y, st);
}

void conv3x3Cat(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
                const float* bias, int Cout, bool relu, void* Y, cudaStream_t st)
{
    const int nt = pickNT(Cout);
    const int colBlocks = Cout / (8 * nt);
    const bf16* a = static_cast<const bf16*>(X1);
    const bf16* b = static_cast<const bf16*>(X2);
    const bf16* w = static_cast<const bf16*>(Wk);
    bf16* y = static_cast<bf16*>(Y);
    if (relu) {
        if (up) launchConv<true, true>(nt, N, H, W, a, C1, b, C2, w, bias, Cout, colBlocks, y, st);
        else launchConv<true, false>(nt, N, H, W, a, C1, b, C2, w, bias, Cout, colBlocks, y, st);
    } else {
        if (up) launchConv<false, true>(nt, N, H, W, a, C1, b, C2, w, bias, Cout, colBlocks, y, st);
        else launchConv<false, false>(nt, N, H, W, a, C1, b, C2, w, bias, Cout, colBlocks, y, st);
    }
}

void convWgrad(const void* X, const void* dY, int N, int H, int W, int Cin, int Cout, float* dW, cudaStream_t st)
{
    const long long total = static_cast<long long>(N) * H * W;
    const int tiles = ((Cout + 63) / 64) * ((Cin + 63) / 64);
    // enough CTAs to fill the GPU a few times over; each reduces >= 256 pixels
    long long splits = (148LL * 8 + 9LL * tiles - 1) / (9LL * tiles);
    long long per = (total + splits - 1) / splits;
    if (per < 256) per = 256;
    per = (per + kWgPix - 1) / kWgPix * kWgPix;
    splits = (total + per - 1) / per;
    kConvWgrad<<<dim3(tiles, 9, static_cast<unsigned>(splits)), 128, 0, st>>>(
        static_cast<const bf16*>(X), static_cast<const bf16*>(dY), N, H, W, Cin, Cout, static_cast<int>(per), dW);
}

void biasGrad(const void* dY, long long pixels, int C, float* db, cudaStream_t st)
{
    if (C % 8 == 0 && C >= 8 && C <= 256) {   // about eight blocks per SM, at least four pixels per thread
        const long long lanes = 256 / (C / 8);
        long long per = (pixels + 148LL * 8 - 1) / (148LL * 8);
        if (per < 4 * lanes) per = 4 * lanes;
        per = (per + lanes - 1) / lanes * lanes;
        const long long ctas = (pixels + per - 1) / per;
        if (ctas > 0)
            kBiasGrad8<<<static_cast<unsigned>(ctas), 256, 0, st>>>(static_cast<const bf16*>(dY), pixels, C, per, db);
        return;
    }
    const int per = 1024;
    const long long ctas = (pixels + per - 1) / per;
    kBiasGrad<<<static_cast<unsigned>(ctas), C / 2, 0, st>>>(static_cast<const bf16*>(dY), pixels, C, per, db);
}

void reluMask(const void* Y, const void* dY, void* out, long long elems, cudaStream_t st)
{
    if (elems % 8 == 0 && reinterpret_cast<uintptr_t>(Y) % 16 == 0 && reinterpret_cast<uintptr_t>(dY) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(out) % 16 == 0) {
        kReluMask8<<<gridFor(elems / 8), 256, 0, st>>>(static_cast<const uint4*>(Y), static_cast<const uint4*>(dY),
                                                        static_cast<uint4*>(out), elems / 8);
        return;
    }
    kReluMask<<<gridFor(elems / 2), 256, 0, st>>>(static_cast<const bf16*>(Y), static_cast<const bf16*>(dY),
                                                  static_cast<bf16*>(out), elems / 2);
}

// a small kernel as a programmatic dependent of the previous kernel in the stream: its blocks may be scheduled
// while a convolution finishes (the convolutions signal their dependents early) and wait in the kernel
template <typename Kernel, typename... Args>
void launchAfterConv(Kernel kernel, int grid, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);   // errors surface through cudaGetLastError
}

void pool2(const void* X, int N, int H, int W, int C, void* Y, cudaStream_t st)
{
    launchAfterConv(kPool2, gridFor(static_cast<long long>(N) * (H / 2) * (W / 2) * (C / 2)), st, static_cast<const bf16*>(X), N,
                    H, W, C, static_cast<bf16*>(Y));
}

void pool2Back(const void* dY, int N, int H, int W, int C, void* dX, cudaStream_t st)
{
    kPool2Back<<<gridFor(static_cast<long long>(N) * H * W * (C / 2)), 256, 0, st>>>(static_cast<const bf16*>(dY), N, H, W,
                                                                                    C, static_cast<bf16*>(dX));
}

void upCat(const void* A, int Ca, const void* B, int Cb, int N, int H, int W, void* out, cudaStream_t st)
{
    kUpCat<<<gridFor(static_cast<long long>(N) * H * W * ((Ca + Cb) / 2)), 256, 0, st>>>(
        static_cast<const bf16*>(A), Ca, static_cast<const bf16*>(B), Cb, N, H, W, static_cast<bf16*>(out));
}

void upsample2(const void* X, int N, int Hs, int Ws, int C, void* Y, cudaStream_t st)
{
    launchAfterConv(kUpsample2, gridFor(static_cast<long long>(N) * Hs * Ws * (C / 8)), st, static_cast<const uint4*>(X), N, Hs,
                    Ws, C / 8, static_cast<uint4*>(Y));
}

void upCatBack(const void* dOut, int Ca, int Cb, int N, int H, int W, void* dA, void* dB, bool addB, cudaStream_t st)
{
    const long long n = static_cast<long long>(N) * (H / 2) * (W / 2) * (Ca / 2) + static_cast<long long>(N) * H * W * (Cb / 2);
    kUpCatBack<<<gridFor(n), 256, 0, st>>>(static_cast<const bf16*>(dOut), Ca, Cb, N, H, W, static_cast<bf16*>(dA),
                                           static_cast<bf16*>(dB), addB ? 1 : 0);
}

void assemble(const float* rad, const float* feat, int N, int H, int W, int Hp, int Wp, void* out, cudaStream_t st)
{
    kAssemble<<<gridFor(static_cast<long long>(N) * Hp * Wp), 256, 0, st>>>(rad, feat, N, H, W, Hp, Wp,
                                                                            static_cast<bf16*>(out));
}

void output(const void* net, const void* in, int N, int H, int W, int Hp, int Wp, float* rad, cudaStream_t st)
{
    launchAfterConv(kOutput, gridFor(static_cast<long long>(N) * H * W), st, static_cast<const bf16*>(net), static_cast<const bf16*>(in),
                    N, H, W, Hp, Wp, rad);
}

void lossL1(const void* net, const void* in, const float* target, long long pixels, void* dNet, float* lossSum,
            cudaStream_t st)
{
    const float scale = 1.0f / static_cast<float>(pixels * 3);
    kLossL1<<<gridFor(pixels), 256, 0, st>>>(static_cast<const bf16*>(net), static_cast<const bf16*>(in), target, pixels,
                                             scale, static_cast<bf16*>(dNet), lossSum);
}

void adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps, float c1,
          float c2, cudaStream_t st)
{
    kAdam<<<gridFor(n), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2);
}

void weightCopies(const float* w, int Cin, int Cout, void* wk, void* wd, cudaStream_t st)
{
    kWeightCopies<<<gridFor(9LL * Cin * Cout), 256, 0, st>>>(w, Cin, Cout, static_cast<bf16*>(wk), static_cast<bf16*>(wd));
}

}  // namespace dn
}  // namespace bte

namespace bte {
namespace dn {

namespace {

// params[4*b ..]: image index, x0, y0, flip bits (1: x, 2: y)
__global__ void kGatherBatch(const float* __restrict__ noisy, const float* __restrict__ feat,
                             const float* __restrict__ target, int width, int height, const int* __restrict__ params,
                             int batch, int crop, float* __restrict__ bRad, float* __restrict__ bFeat,
                             float* __restrict__ bTarget)
{
    const long long total = static_cast<long long>(batch) * crop * crop;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % crop);
        const long long r = i / crop;
        const int y = static_cast<int>(r % crop);
        const int b = static_cast<int>(r / crop);
        const int img = params[4 * b], x0 = params[4 * b + 1], y0 = params[4 * b + 2], fl = params[4 * b + 3];
        const int sx = x0 + ((fl & 1) ? crop - 1 - x : x);
        const int sy = y0 + ((fl & 2) ? crop - 1 - y : y);
        const size_t src = (static_cast<size_t>(img) * height + sy) * width + sx;
        for (int c = 0; c < 3; ++c) {
            bRad[3 * i + c] = noisy[3 * src + c];
            bTarget[3 * i + c] = target[3 * src + c];
        }
        for (int c = 0; c < 6; ++c) bFeat[6 * i + c] = feat[6 * src + c];
    }
}

}  // namespace

void gatherBatch(const float* noisy, const float* feat, const float* target, int width, int height, const int* params,
                 int batch, int crop, float* bRad, float* bFeat, float* bTarget, cudaStream_t st)
{
    const long long n = static_cast<long long>(batch) * crop * crop;
    const int g = static_cast<int>((n + 255) / 256 < 148 * 32 ? (n + 255) / 256 : 148 * 32);
    kGatherBatch<<<g, 256, 0, st>>>(noisy, feat, target, width, height, params, batch, crop, bRad, bFeat, bTarget);
}

}  // namespace dn
}  // namespace bte
