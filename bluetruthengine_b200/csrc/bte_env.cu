// bte_env.cu -- environment-map sampling tables on the GPU.
//
// CDF mode (bit-exact with the reference): the marginal/conditional CDF of
// src/host/scene_upload.cu:422-459 -- per row an FP32 sequential prefix sum
// of luminance * sin(theta_row), then the FP32 prefix of the row sums.  Each
// row is one thread summing in the reference's order; sin(theta_row) comes
// from the host, computed exactly as the reference computes it.
//
// Alias mode: the same weights evaluated in FP64, row sums and the total in
// FP64, one alias table per row (columns) and one over rows (M. D. Vose's
// linear-time construction, IEEE TSE 17(9) 1991), plus the per-pixel discrete
// probability used for MIS.  Sampling is then O(1) per NEE instead of two
// binary searches.
#include "bte_internal.h"
#include "bte_kernels.h"
#include "bte_math.cuh"

#include <cstdint>
#include <mutex>
#include <string>

namespace bte {

namespace {

__global__ void kEnvCdfRows(const float4* __restrict__ tex, int w, int h, const float* __restrict__ sinTheta, float* cond)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    if (iy >= h) return;
    const float st = sinTheta[iy];
    float* row = cond + static_cast<size_t>(iy) * (w + 1);
    float run = 0.0f;
    row[0] = 0.0f;
    for (int ix = 0; ix < w; ++ix) {
        const float4 t = tex[static_cast<size_t>(iy) * w + ix];
        const float lum = 0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z;
        run = run + lum * st;
        row[ix + 1] = run;
    }
}

__global__ void kEnvCdfMarginal(const float* __restrict__ cond, int w, int h, float* marg)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    float run = 0.0f;
    marg[0] = 0.0f;
    for (int iy = 0; iy < h; ++iy) {
        run = run + cond[static_cast<size_t>(iy) * (w + 1) + w];
        marg[iy + 1] = run;
    }
}

__global__ void kEnvWeights(const float4* __restrict__ tex, int w, int h, double* wt, double* rowSum)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    if (iy >= h) return;
    const double theta = m::kPi * (static_cast<double>(iy) + 0.5) / static_cast<double>(h);
    const double st = m::sinD(theta);
    double rs = 0.0;
    for (int ix = 0; ix < w; ++ix) {
        const float4 t = tex[static_cast<size_t>(iy) * w + ix];
        const double lum = 0.2126 * static_cast<double>(t.x) + 0.7152 * static_cast<double>(t.y) +
                           0.0722 * static_cast<double>(t.z);
        const double v = lum * st;
        wt[static_cast<size_t>(iy) * w + ix] = v;
        rs += v;
    }
    rowSum[iy] = rs;
}

__device__ void voseBuild(const double* wts, int n, double sum, float* prob, int* alias, int* small, int* large,
                          double* scaled)
{
    int ns = 0, nl = 0;
    if (!(sum > 0.0)) {
        for (int i = 0; i < n; ++i) { prob[i] = 1.0f; alias[i] = i; }
        return;
    }
    for (int i = 0; i < n; ++i) {
        scaled[i] = wts[i] * static_cast<double>(n) / sum;
        if (scaled[i] < 1.0) small[ns++] = i;
        else large[nl++] = i;
    }
    while (ns > 0 && nl > 0) {
        const int l = small[--ns];
        const int g = large[--nl];
        prob[l] = static_cast<float>(scaled[l]);
        alias[l] = g;
        scaled[g] = (scaled[g] + scaled[l]) - 1.0;
        if (scaled[g] < 1.0) small[ns++] = g;
        else large[nl++] = g;
    }
    while (nl > 0) { const int g = large[--nl]; prob[g] = 1.0f; alias[g] = g; }
    while (ns > 0) { const int l = small[--ns]; prob[l] = 1.0f; alias[l] = l; }
}

__global__ void kEnvTotal(const double* rowSum, int h, double* total)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double t = 0.0;
    for (int iy = 0; iy < h; ++iy) t += rowSum[iy];
    *total = t;
}

// scratch: small/large/scaled work lists, w entries per row
__global__ void kEnvAliasRows(const double* __restrict__ wt, const double* __restrict__ rowSum, int w, int h,
                              const double* __restrict__ total, float* colProb, int* colAlias, float* pixelPdf,
                              int* scratchI, double* scratchD)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    if (iy >= h) return;
    const size_t off = static_cast<size_t>(iy) * w;
    voseBuild(wt + off, w, rowSum[iy], colProb + off, colAlias + off, scratchI + 2 * off, scratchI + 2 * off + w,
              scratchD + off);
    const double T = *total;
    for (int ix = 0; ix < w; ++ix)
        pixelPdf[off + ix] = (T > 0.0) ? static_cast<float>(wt[off + ix] / T) : 0.0f;
}

__global__ void kEnvAliasMarginal(const double* rowSum, int h, const double* total, float* rowProb, int* rowAlias,
                                  int* scratchI, double* scratchD)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    voseBuild(rowSum, h, *total, rowProb, rowAlias, scratchI, scratchI + h, scratchD);
}

}  // namespace

#define ENV_CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { err = std::string("env tables: ") + cudaGetErrorString(e_); rc = -1; goto done; } } while (0)

int buildEnvCdf(const float4* dTexels, int w, int h, const float* hSinTheta, float* dMarginal, float* dConditional,
                cudaStream_t st, std::string& err)
{
    int rc = 0;
    float* dSin = nullptr;
    ENV_CK(cudaMalloc(&dSin, sizeof(float) * h));
    ENV_CK(cudaMemcpyAsync(dSin, hSinTheta, sizeof(float) * h, cudaMemcpyHostToDevice, st));
    kEnvCdfRows<<<(h + 127) / 128, 128, 0, st>>>(dTexels, w, h, dSin, dConditional);
    kEnvCdfMarginal<<<1, 1, 0, st>>>(dConditional, w, h, dMarginal);
    ENV_CK(cudaGetLastError());
    ENV_CK(cudaStreamSynchronize(st));
done:
    cudaFree(dSin);
    return rc;
}

int buildEnvAlias(const float4* dTexels, int w, int h, float* dRowProb, int* dRowAlias, float* dColProb, int* dColAlias,
                  float* dPixelPdf, double* hTotal, cudaStream_t st, std::string& err)
{
    int rc = 0;
    double *wt = nullptr, *rowSum = nullptr, *total = nullptr, *scratchD = nullptr;
    int* scratchI = nullptr;
    const size_t n = static_cast<size_t>(w) * h;
    ENV_CK(cudaMalloc(&wt, sizeof(double) * n));
    ENV_CK(cudaMalloc(&rowSum, sizeof(double) * h));
    ENV_CK(cudaMalloc(&total, sizeof(double)));
    ENV_CK(cudaMalloc(&scratchD, sizeof(double) * (n > static_cast<size_t>(h) ? n : h)));
    ENV_CK(cudaMalloc(&scratchI, sizeof(int) * 2 * (n > static_cast<size_t>(h) ? n : h)));
    kEnvWeights<<<(h + 127) / 128, 128, 0, st>>>(dTexels, w, h, wt, rowSum);
    kEnvTotal<<<1, 1, 0, st>>>(rowSum, h, total);
    kEnvAliasRows<<<(h + 127) / 128, 128, 0, st>>>(wt, rowSum, w, h, total, dColProb, dColAlias, dPixelPdf, scratchI,
                                                   scratchD);
    ENV_CK(cudaGetLastError());
    ENV_CK(cudaStreamSynchronize(st));
    kEnvAliasMarginal<<<1, 1, 0, st>>>(rowSum, h, total, dRowProb, dRowAlias, scratchI, scratchD);
    ENV_CK(cudaGetLastError());
    ENV_CK(cudaMemcpyAsync(hTotal, total, sizeof(double), cudaMemcpyDeviceToHost, st));
    ENV_CK(cudaStreamSynchronize(st));
done:
    cudaFree(wt); cudaFree(rowSum); cudaFree(total); cudaFree(scratchD); cudaFree(scratchI);
    return rc;
}

}  // namespace bte

// ---------------------------------------------------------------- no-allocation variant
//
// bte_env_build_alias_noalloc builds the same FP64 alias tables as the
// allocating path above, but never calls cudaMalloc/cudaFree (or anything that
// allocates).  It exists for callers that cannot allocate device memory at the
// moment they need new tables: a render loop that swaps environment maps
// between frames (cudaMalloc and cudaFree synchronise the whole device and
// would stall the frames already queued), and host applications that reserve
// all device memory for their own pool up front, leaving nothing for a
// library to allocate from.  The caller owns the input texels and every output
// table; the intermediate FP64 weights, row sums and Vose work lists live in
// one file-scope device array of fixed size, so maps are limited to
// kNoAllocMaxTexels texels and kNoAllocMaxRows rows.
//
// The first use of the array on a device looks up its device address; under
// CUDA's lazy module loading that lookup also loads this file's module, which
// is when the array's memory is taken.  The renderer's device initialisation
// (any bte_* call that sets up the renderer) does this lookup, and so does the
// first call here: a caller that reserves the rest of device memory for its
// own pool should make one of those calls first, and the first call here
// should come before any stream capture.
//
// The array is shared by every call in the process: two calls whose kernels
// overlap on the GPU (different streams, or different host threads on one
// device) race on it and produce garbage; serialise them.  Nothing in it has
// to start at zero -- every scratch word is written before it is read -- and
// it keeps whatever the last call left there.  Each device that loads the
// library holds the array until the process exits.
namespace bte {
namespace {

constexpr int kNoAllocMaxTexels = 512 * 256;
constexpr int kNoAllocMaxRows = 4096;
constexpr size_t kAlign = 256;
constexpr size_t alignUp(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
// layout: weights [texels] double | row sums [rows] double | work ints [2*texels] | work doubles [texels]
constexpr size_t kOffWeights = 0;
constexpr size_t kOffRowSum = alignUp(kOffWeights + sizeof(double) * kNoAllocMaxTexels);
constexpr size_t kOffWorkI = alignUp(kOffRowSum + sizeof(double) * kNoAllocMaxRows);
constexpr size_t kOffWorkD = alignUp(kOffWorkI + sizeof(int) * 2 * kNoAllocMaxTexels);
constexpr size_t kNoAllocScratchBytes = alignUp(kOffWorkD + sizeof(double) * kNoAllocMaxTexels);

static __device__ __align__(256) unsigned char g_envAliasScratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_scratchAddr[kMaxDevices] = {};
std::mutex g_scratchMutex;

// Device address of g_envAliasScratch on the current device, looked up once per
// device (the host-side symbol is a stand-in, not a device address).
int scratchForCurrentDevice(unsigned char** out, std::string& err)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return -1; }
    if (dev < 0 || dev >= kMaxDevices) { err = "device ordinal out of range"; return -1; }
    std::lock_guard<std::mutex> lk(g_scratchMutex);
    if (!g_scratchAddr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_envAliasScratch);
        if (e != cudaSuccess || !p) {
            err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return -1;
        }
        g_scratchAddr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratchAddr[dev];
    return 0;
}

}  // namespace

// Looks up (and, under lazy module loading, loads) the scratch array on the current device.  The renderer's
// device initialisation calls it, so a caller that initialises the renderer before reserving its memory pool
// has the array in place before its first bte_env_build_alias_noalloc.
int prepareEnvNoallocScratch(std::string& err)
{
    unsigned char* base = nullptr;
    return scratchForCurrentDevice(&base, err);
}

}  // namespace bte

extern "C" int bte_env_build_alias_noalloc(const float* dTexelsRGBA, int width, int height, float* dRowProb,
                                           int* dRowAlias, float* dColProb, int* dColAlias, float* dPixelPdf,
                                           double* dTotalPower, void* stream)
{
    using namespace bte;
    if (!dTexelsRGBA || !dRowProb || !dRowAlias || !dColProb || !dColAlias || !dPixelPdf || !dTotalPower) {
        setError("bte_env_build_alias_noalloc: null pointer argument");
        return -1;
    }
    if (width <= 0 || height <= 0) {
        setError("bte_env_build_alias_noalloc: width and height must be positive");
        return -1;
    }
    if (static_cast<long long>(width) * height > kNoAllocMaxTexels || height > kNoAllocMaxRows) {
        setError("bte_env_build_alias_noalloc: " + std::to_string(width) + "x" + std::to_string(height) +
                 " exceeds the fixed scratch of this entry point (at most " + std::to_string(kNoAllocMaxTexels) +
                 " texels and " + std::to_string(kNoAllocMaxRows) + " rows); use bte_init_env_map for larger maps");
        return -1;
    }
    if (reinterpret_cast<uintptr_t>(dTexelsRGBA) % 16 != 0) {
        setError("bte_env_build_alias_noalloc: texels must be 16-byte aligned (float4 per texel)");
        return -1;
    }
    if (reinterpret_cast<uintptr_t>(dTotalPower) % 8 != 0 || reinterpret_cast<uintptr_t>(dRowProb) % 4 != 0 ||
        reinterpret_cast<uintptr_t>(dRowAlias) % 4 != 0 || reinterpret_cast<uintptr_t>(dColProb) % 4 != 0 ||
        reinterpret_cast<uintptr_t>(dColAlias) % 4 != 0 || reinterpret_cast<uintptr_t>(dPixelPdf) % 4 != 0) {
        setError("bte_env_build_alias_noalloc: dTotalPower must be 8-byte aligned and the tables 4-byte aligned");
        return -1;
    }
    unsigned char* base = nullptr;
    std::string err;
    if (scratchForCurrentDevice(&base, err) != 0) {
        setError("bte_env_build_alias_noalloc: " + err);
        return -1;
    }
    double* wt = reinterpret_cast<double*>(base + kOffWeights);
    double* rowSum = reinterpret_cast<double*>(base + kOffRowSum);
    int* workI = reinterpret_cast<int*>(base + kOffWorkI);
    double* workD = reinterpret_cast<double*>(base + kOffWorkD);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float4* tex = reinterpret_cast<const float4*>(dTexelsRGBA);
    kEnvWeights<<<(height + 127) / 128, 128, 0, st>>>(tex, width, height, wt, rowSum);
    kEnvTotal<<<1, 1, 0, st>>>(rowSum, height, dTotalPower);
    kEnvAliasRows<<<(height + 127) / 128, 128, 0, st>>>(wt, rowSum, width, height, dTotalPower, dColProb, dColAlias,
                                                        dPixelPdf, workI, workD);
    kEnvAliasMarginal<<<1, 1, 0, st>>>(rowSum, height, dTotalPower, dRowProb, dRowAlias, workI, workD);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        setError(std::string("bte_env_build_alias_noalloc: ") + cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
