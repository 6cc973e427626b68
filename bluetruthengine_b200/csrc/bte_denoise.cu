// bte_denoise.cu -- the learned denoiser: a 5-level U-Net over the noisy
// radiance and the albedo/normal features, trained on image pairs
// this renderer produces, replacing the reference's vendor denoiser stage
// (src/host/denoiser.cu:72-109, cudaToggleDenoiser render_kernel.h:187).
//
// Network (3x3 convolutions, ReLU, 2x2 average pooling, nearest upsampling
// with skip concatenation), channels per level 32/48/64/96/128:
//   input 16 ch = log(1 + L) (3), albedo (3), normal (3), zeros (7)
//   encoder: 2 convs per level, pool between levels
//   decoder: upsample + concatenate the encoder output of the level, 2 convs
//   output conv 32 -> 16 (3 used), no activation, added to the input log radiance
// Weights are FP32 masters updated by Adam; the convolutions run in BF16 on
// the tensor cores with FP32 accumulation.  Training samples random crops
// (with flips) of a device-resident image set and minimises the L1 error of
// log(1 + L) against the long-run targets.
#include "bte_denoise.h"
#include "bte_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iterator>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace bte {
namespace dn {
namespace {

struct Conv { int cin, cout, cinLogical; bool relu; };
enum Op { kConvOp, kPoolOp, kUpCatOp };
struct Step { Op op; int src, src2, dst, conv; };
struct TensorSpec { int c, level; };

// tensors: 0 in | 1 e0a 2 e0b | 3 p1 4 e1a 5 e1b | 6 p2 7 e2a 8 e2b | 9 p3 10 e3a 11 e3b | 12 p4 13 e4a 14 e4b |
//          15 c3 16 d3a 17 d3b | 18 c2 19 d2a 20 d2b | 21 c1 22 d1a 23 d1b | 24 c0 25 d0a 26 d0b | 27 out
const TensorSpec kTensors[] = {
    {16, 0}, {32, 0}, {32, 0}, {32, 1}, {48, 1}, {48, 1}, {48, 2}, {64, 2}, {64, 2}, {64, 3}, {96, 3}, {96, 3},
    {96, 4}, {128, 4}, {128, 4}, {224, 3}, {96, 3}, {96, 3}, {160, 2}, {64, 2}, {64, 2}, {112, 1}, {48, 1}, {48, 1},
    {80, 0}, {32, 0}, {32, 0}, {16, 0}};
constexpr int kTensorCount = 28;
const Conv kConvs[] = {
    {16, 32, 9, true},   {32, 32, 32, true},   {32, 48, 32, true},  {48, 48, 48, true}, {48, 64, 48, true},
    {64, 64, 64, true},  {64, 96, 64, true},   {96, 96, 96, true},  {96, 128, 96, true}, {128, 128, 128, true},
    {224, 96, 224, true}, {96, 96, 96, true},  {160, 64, 160, true}, {64, 64, 64, true}, {112, 48, 112, true},
    {48, 48, 48, true},  {80, 32, 80, true},   {32, 32, 32, true},  {32, 16, 32, false}};
constexpr int kConvCount = 19;
const Step kSteps[] = {
    {kConvOp, 0, -1, 1, 0},   {kConvOp, 1, -1, 2, 1},   {kPoolOp, 2, -1, 3, -1},  {kConvOp, 3, -1, 4, 2},
    {kConvOp, 4, -1, 5, 3},   {kPoolOp, 5, -1, 6, -1},  {kConvOp, 6, -1, 7, 4},   {kConvOp, 7, -1, 8, 5},
    {kPoolOp, 8, -1, 9, -1},  {kConvOp, 9, -1, 10, 6},  {kConvOp, 10, -1, 11, 7}, {kPoolOp, 11, -1, 12, -1},
    {kConvOp, 12, -1, 13, 8}, {kConvOp, 13, -1, 14, 9}, {kUpCatOp, 14, 11, 15, -1}, {kConvOp, 15, -1, 16, 10},
    {kConvOp, 16, -1, 17, 11}, {kUpCatOp, 17, 8, 18, -1}, {kConvOp, 18, -1, 19, 12}, {kConvOp, 19, -1, 20, 13},
    {kUpCatOp, 20, 5, 21, -1}, {kConvOp, 21, -1, 22, 14}, {kConvOp, 22, -1, 23, 15}, {kUpCatOp, 23, 2, 24, -1},
    {kConvOp, 24, -1, 25, 16}, {kConvOp, 25, -1, 26, 17}, {kConvOp, 26, -1, 27, 18}};
constexpr int kStepCount = sizeof(kSteps) / sizeof(kSteps[0]);
constexpr int kLevels = 5;
constexpr int kAlign = 1 << (kLevels - 1);   // image sizes are padded to a multiple of 16

struct CudaErr { std::string msg; };
void ck(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw CudaErr{std::string(what) + ": " + cudaGetErrorString(e)};
}

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n)
    {
        if (bytes >= n && p) return;
        release();
        ck(cudaMalloc(&p, n), "cudaMalloc");
        bytes = n;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct Net {
    bool ready = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // parameters: per conv [9][cout][cin] weights then [cout] bias, FP32
    size_t wOff[kConvCount] = {}, bOff[kConvCount] = {}, bfOff[kConvCount] = {};
    size_t paramCount = 0, bfCount = 0;
    Buf w, grad, m, v, wk, wd;
    long long adamStep = 0;
    // activations for one (N, Hp, Wp)
    int aN = 0, aHp = 0, aWp = 0;
    bool aGrad = false;
    Buf act[kTensorCount], gact[kTensorCount];
    Buf rad, feat, target, out, lossSum, params;
    // training set (device)
    Buf dsNoisy, dsFeat, dsTarget;
    int dsCount = 0, dsW = 0, dsH = 0;
    float lastMs = 0.0f;
    int tcMode = 2;   // convolution kernels: 0 warp-level mma.sync only, 1 tcgen05 pixel tiles, 2/3 tcgen05 row tiles
    int wgradKind = 1;   // weight gradients: 1 tcgen05 where the shape allows (default), 0 warp-level mma.sync,
                         // 2.. tcgen05 with pipeline shape wgradKind - 1 (convWgradTc's variants)
    Buf wgScratch;       // channel-major copies for the tcgen05 weight gradient
    Buf errFlag;          // set by a tcgen05 convolution that timed out
    Buf rowScratch;       // FP32 partial sums of a row-tile convolution that runs in passes
    Buf upBuf;            // a decoder layer's upsampled input at full resolution (row-tile kernel)
    unsigned allocGen = 0;   // bumped whenever a buffer the inference graph refers to is (re)allocated
    // inference sequence (assemble, convolutions, output) captured in a CUDA graph for one shape, kernel
    // choice and set of buffers; replayed while all of them stay the same
    cudaGraphExec_t fwdExec = nullptr;
    int fwdKey[7] = {};
    const void* fwdPtrs[7] = {};
};

Net net;
std::mutex netMutex;
std::string lastErr;

void setupLayout()
{
    size_t off = 0, bo = 0;
    for (int i = 0; i < kConvCount; ++i) {
        net.wOff[i] = off;
        off += 9ull * kConvs[i].cin * kConvs[i].cout;
        net.bOff[i] = off;
        off += kConvs[i].cout;
        net.bfOff[i] = bo;
        bo += (9ull * kConvs[i].cin * kConvs[i].cout + 127) / 128 * 128;   // 256-byte aligned bf16 slices
    }
    net.paramCount = off;
    net.bfCount = bo;
}

void refreshCopies()
{
    for (int i = 0; i < kConvCount; ++i)
        weightCopies(net.w.as<float>() + net.wOff[i], kConvs[i].cin, kConvs[i].cout,
                     net.wk.as<unsigned short>() + net.bfOff[i], net.wd.as<unsigned short>() + net.bfOff[i], net.stream);
}

void ensureNet()
{
    if (net.stream) return;
    net.errFlag.ensure(sizeof(unsigned int));
    ck(cudaMemset(net.errFlag.p, 0, sizeof(unsigned int)), "cudaMemset");
    ck(cudaStreamCreateWithFlags(&net.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreate(&net.ev0), "cudaEventCreate");
    ck(cudaEventCreate(&net.ev1), "cudaEventCreate");
    setupLayout();
}

void initParams(uint64_t seed)
{
    ensureNet();
    std::vector<float> h(net.paramCount, 0.0f);
    std::mt19937_64 rng(seed);
    for (int i = 0; i < kConvCount; ++i) {
        const Conv& c = kConvs[i];
        // He initialisation over the logical fan-in; padded input channels and
        // unused output channels stay zero (their gradients are zero as well)
        const double sd = std::sqrt(2.0 / (9.0 * c.cinLogical)) * (c.relu ? 1.0 : 0.1);
        std::normal_distribution<double> nd(0.0, sd);
        const int coutUsed = (i == kConvCount - 1) ? 3 : c.cout;
        for (int tap = 0; tap < 9; ++tap)
            for (int co = 0; co < c.cout; ++co)
                for (int ci = 0; ci < c.cin; ++ci) {
                    const double r = nd(rng);
                    if (co < coutUsed && ci < c.cinLogical)
                        h[net.wOff[i] + (static_cast<size_t>(tap) * c.cout + co) * c.cin + ci] = static_cast<float>(r);
                }
    }
    net.w.ensure(net.paramCount * 4);
    net.grad.ensure(net.paramCount * 4);
    net.m.ensure(net.paramCount * 4);
    net.v.ensure(net.paramCount * 4);
    net.wk.ensure(net.bfCount * 2);
    net.wd.ensure(net.bfCount * 2);
    ck(cudaMemcpyAsync(net.w.p, h.data(), net.paramCount * 4, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
    ck(cudaMemsetAsync(net.m.p, 0, net.paramCount * 4, net.stream), "cudaMemsetAsync");
    ck(cudaMemsetAsync(net.v.p, 0, net.paramCount * 4, net.stream), "cudaMemsetAsync");
    ck(cudaMemsetAsync(net.wk.p, 0, net.bfCount * 2, net.stream), "cudaMemsetAsync");
    ck(cudaMemsetAsync(net.wd.p, 0, net.bfCount * 2, net.stream), "cudaMemsetAsync");
    refreshCopies();
    ck(cudaStreamSynchronize(net.stream), "init");
    net.adamStep = 0;
    net.ready = true;
}

void ensureActs(int N, int Hp, int Wp, bool withGrad)
{
    if (net.aN == N && net.aHp == Hp && net.aWp == Wp && (net.aGrad || !withGrad)) return;
    for (int t = 0; t < kTensorCount; ++t) {
        const size_t elems = static_cast<size_t>(N) * (Hp >> kTensors[t].level) * (Wp >> kTensors[t].level) * kTensors[t].c;
        net.act[t].release();
        net.act[t].ensure(elems * 2);
        net.gact[t].release();
        if (withGrad) net.gact[t].ensure(elems * 2);
    }
    net.aN = N; net.aHp = Hp; net.aWp = Wp; net.aGrad = withGrad;
    ++net.allocGen;
}

// One 3x3 convolution over concat(up ? upsample(X1) : X1, X2).  tcMode 2: layers with at least 32
// 128-pixel row tiles (64 if they run in passes) and Cout 16..64, 96 or 128 go to the tcgen05 row-tile kernel (in passes over
// the input channels where weights and slabs do not fit shared memory at once); tcMode 1: layers that
// fill the machine four times over with 128-pixel tiles go to the pixel-tile kernel; the rest to the
// warp-level kernel.  force: -1 by tcMode, 0 warp-level, 1 pixel tiles, 2 row tiles.
// pool (optional, row tiles only): also write the 2x2 average pool of Y there if the kernel can; returns
// whether it did.
bool convDispatch(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
                  const float* bias, int Cout, bool relu, void* Y, cudaStream_t st, int force = -1, void* pool = nullptr)
{
    const long long px = static_cast<long long>(N) * H * W;
    int kind = force;
    if (kind < 0) {
        kind = 0;
        const long long rowTiles = static_cast<long long>(N) * H * ((W + 127) / 128);
        // a layer that runs in passes pays one launch per pass: it needs twice the tiles of a one-pass layer
        const bool passes = convTcRowScratchBytes(C1, C2, up, Cout, N, H, W) > 0;
        if ((net.tcMode == 2 || net.tcMode == 3) && rowTiles >= (passes ? 64 : 32) && convTcRowSupported(C1, C2, up, Cout)) kind = 2;
        else if (net.tcMode == 1 && px >= 128LL * 148 * 4 && convTcSupported(C1 + C2, Cout)) kind = 1;
    }
    if (kind == 2 && !convTcRowSupported(C1, C2, up, Cout))
        throw CudaErr{"denoiser: the tcgen05 row-tile kernel does not take this layer (Cout 16/32/48/64/96/128, Cin in 16-channel passes)"};
    if (kind == 1 && !convTcSupported(C1 + C2, Cout))
        throw CudaErr{"denoiser: the tcgen05 pixel-tile kernel does not take this layer"};
    if (kind == 2 && up && net.tcMode != 3) {
        // the row-tile kernel reads an upsampled input fastest as a full-resolution tensor: upsample it first (one
        // HBM pass) instead of expanding the half-resolution slab in shared memory per tile (measured over the
        // network at 1080p: 1.205 ms against 1.24 ms; mode 3 keeps the in-kernel expansion)
        const size_t need = static_cast<size_t>(N) * H * W * C1 * 2;
        if (net.upBuf.bytes < need || !net.upBuf.p) {
            net.upBuf.ensure(need);
            ++net.allocGen;
        }
        upsample2(X1, N, H / 2, W / 2, C1, net.upBuf.p, st);
        X1 = net.upBuf.p;
        up = false;
    }
    if (kind == 2) {
        const size_t scratch = convTcRowScratchBytes(C1, C2, up, Cout, N, H, W);
        if (scratch && (net.rowScratch.bytes < scratch || !net.rowScratch.p)) {
            net.rowScratch.ensure(scratch);
            ++net.allocGen;
        }
        return conv3x3TcRow(X1, C1, up, X2, C2, N, H, W, Wk, bias, Cout, relu, Y, scratch ? net.rowScratch.p : nullptr, pool,
                            net.errFlag.as<unsigned int>(), st);
    }
    if (kind == 1) conv3x3Tc(X1, C1, up, X2, C2, N, H, W, Wk, bias, Cout, relu, Y, net.errFlag.as<unsigned int>(), st);
    else conv3x3Cat(X1, C1, up, X2, C2, N, H, W, Wk, bias, Cout, relu, Y, st);
    return false;
}

void checkTcFlag()
{
    unsigned int f = 0;
    ck(cudaMemcpyAsync(&f, net.errFlag.p, sizeof(f), cudaMemcpyDeviceToHost, net.stream), "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(net.stream), "sync");
    if (f) {
        ck(cudaMemsetAsync(net.errFlag.p, 0, sizeof(f), net.stream), "cudaMemsetAsync");
        throw CudaErr{"denoiser: a tensor-core convolution timed out waiting for its pipeline"};
    }
}

// Training keeps the concatenated decoder inputs (the weight gradients read
// them); inference lets the decoder convolutions read upsample + skip in place.
void forward(int N, int Hp, int Wp, bool training)
{
    cudaStream_t st = net.stream;
    for (int k = 0; k < kStepCount; ++k) {
        const Step& s = kSteps[k];
        const TensorSpec& ts = kTensors[s.src];
        const int H = Hp >> ts.level, W = Wp >> ts.level;
        if (s.op == kConvOp) {
            const Conv& c = kConvs[s.conv];
            const Step* prev = k > 0 ? &kSteps[k - 1] : nullptr;
            if (!training && prev && prev->op == kUpCatOp && prev->dst == s.src) {
                const TensorSpec& low = kTensors[prev->src];
                const TensorSpec& skip = kTensors[prev->src2];
                convDispatch(net.act[prev->src].p, low.c, true, net.act[prev->src2].p, skip.c, N, H, W,
                             net.wk.as<unsigned short>() + net.bfOff[s.conv], net.w.as<float>() + net.bOff[s.conv], c.cout,
                             c.relu, net.act[s.dst].p, st);
            } else {
                // an inference conv whose output feeds the next step's pool may write the pool in its epilogue
                const Step* next = k + 1 < kStepCount ? &kSteps[k + 1] : nullptr;
                const bool fuse = !training && next && next->op == kPoolOp && next->src == s.dst;
                if (convDispatch(net.act[s.src].p, c.cin, false, nullptr, 0, N, H, W,
                                 net.wk.as<unsigned short>() + net.bfOff[s.conv], net.w.as<float>() + net.bOff[s.conv], c.cout,
                                 c.relu, net.act[s.dst].p, st, -1, fuse ? net.act[next->dst].p : nullptr))
                    ++k;   // the pool step is done
            }
        } else if (s.op == kPoolOp) {
            pool2(net.act[s.src].p, N, H, W, ts.c, net.act[s.dst].p, st);
        } else if (training) {
            const TensorSpec& skip = kTensors[s.src2];
            upCat(net.act[s.src].p, ts.c, net.act[s.src2].p, skip.c, N, Hp >> skip.level, Wp >> skip.level,
                  net.act[s.dst].p, st);
        }
    }
}

// gradient of the network output is in gact[27]
void backward(int N, int Hp, int Wp)
{
    cudaStream_t st = net.stream;
    ck(cudaMemsetAsync(net.grad.p, 0, net.paramCount * 4, st), "cudaMemsetAsync");
    for (int k = kStepCount - 1; k >= 0; --k) {
        const Step& s = kSteps[k];
        const TensorSpec& ts = kTensors[s.src];
        const int H = Hp >> ts.level, W = Wp >> ts.level;
        if (s.op == kConvOp) {
            const Conv& c = kConvs[s.conv];
            const long long elems = static_cast<long long>(N) * H * W * c.cout;
            if (c.relu) reluMask(net.act[s.dst].p, net.gact[s.dst].p, net.gact[s.dst].p, elems, st);
            if (net.wgradKind >= 1 && convWgradTcSupported(N, H, W, c.cin, c.cout)) {
                net.wgScratch.ensure(convWgradTcScratchBytes(N, H, W, c.cin, c.cout));
                convWgradTc(net.act[s.src].p, net.gact[s.dst].p, N, H, W, c.cin, c.cout,
                            net.grad.as<float>() + net.wOff[s.conv], net.wgScratch.p, net.errFlag.as<unsigned int>(), st,
                            net.wgradKind - 1);
            } else {
                convWgrad(net.act[s.src].p, net.gact[s.dst].p, N, H, W, c.cin, c.cout,
                          net.grad.as<float>() + net.wOff[s.conv], st);
            }
            biasGrad(net.gact[s.dst].p, static_cast<long long>(N) * H * W, c.cout, net.grad.as<float>() + net.bOff[s.conv], st);
            if (s.src != 0)
                convDispatch(net.gact[s.dst].p, c.cout, false, nullptr, 0, N, H, W,
                             net.wd.as<unsigned short>() + net.bfOff[s.conv], nullptr, c.cin, false, net.gact[s.src].p, st);
        } else if (s.op == kPoolOp) {
            // the pooled tensor's other consumer (the decoder concatenation) wrote its gradient already
            pool2Back(net.gact[s.dst].p, N, H, W, ts.c, net.gact[s.src].p, st);
        } else {
            const TensorSpec& skip = kTensors[s.src2];
            upCatBack(net.gact[s.dst].p, ts.c, skip.c, N, Hp >> skip.level, Wp >> skip.level, net.gact[s.src].p,
                      net.gact[s.src2].p, false, st);
        }
    }
}

int padTo(int x) { return (x + kAlign - 1) / kAlign * kAlign; }

template <typename F>
int guardedDn(F&& fn)
{
    std::lock_guard<std::mutex> lk(netMutex);
    try {
        return fn();
    } catch (const CudaErr& e) {
        lastErr = e.msg;
        setError(e.msg);
        return -1;
    } catch (const std::exception& e) {
        lastErr = e.what();
        setError(lastErr);
        return -1;
    }
}

}  // namespace

namespace {

void inferenceSequence(const float* dRad, const float* dFeat, int N, int H, int W, int Hp, int Wp, float* dOut, cudaStream_t st)
{
    assemble(dRad, dFeat, N, H, W, Hp, Wp, net.act[0].p, st);
    forward(N, Hp, Wp, false);
    output(net.act[27].p, net.act[0].p, N, H, W, Hp, Wp, dOut, st);
}

// Capture the sequence just run eagerly (buffers already allocated) for the next calls with the same key;
// on any failure the denoiser simply stays eager.
void captureInference(const float* dRad, const float* dFeat, int N, int H, int W, int Hp, int Wp, float* dOut,
                      const int (&key)[7], const void* const (&ptrs)[7])
{
    if (net.fwdExec) {
        cudaGraphExecDestroy(net.fwdExec);
        net.fwdExec = nullptr;
    }
    cudaStream_t st = net.stream;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    bool ok = true;
    try {
        inferenceSequence(dRad, dFeat, N, H, W, Hp, Wp, dOut, st);
    } catch (...) {
        ok = false;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    cudaGraphExec_t exec = nullptr;
    if (ok && e == cudaSuccess && g && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
        net.fwdExec = exec;
        std::copy(std::begin(key), std::end(key), net.fwdKey);
        std::copy(std::begin(ptrs), std::end(ptrs), net.fwdPtrs);
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
}

}  // namespace

// Denoise [N, H, W] radiance (+ features) held on the device into `outRad`.  The first call for a shape runs
// eagerly and captures the sequence in a CUDA graph; later calls with the same shape, kernel choice and
// buffers replay it (no per-kernel host work).
void denoiseDevice(const float* dRad, const float* dFeat, int N, int H, int W, float* dOut, cudaStream_t waitOn)
{
    if (!net.ready) throw CudaErr{"denoiser: no weights (bte_denoiser_init / bte_denoiser_set_params)"};
    const int Hp = padTo(H), Wp = padTo(W);
    ensureActs(N, Hp, Wp, false);
    cudaStream_t st = net.stream;
    if (waitOn) {
        ck(cudaEventRecord(net.ev0, waitOn), "cudaEventRecord");
        ck(cudaStreamWaitEvent(st, net.ev0, 0), "cudaStreamWaitEvent");
    }
    const int key[7] = {N, H, W, Hp, Wp, net.tcMode, static_cast<int>(net.allocGen)};
    const void* const ptrs[7] = {dRad, dFeat, dOut, net.act[0].p, net.wk.p, net.w.p, net.rowScratch.p};
    const bool replay = net.fwdExec && std::equal(std::begin(key), std::end(key), net.fwdKey) &&
                        std::equal(std::begin(ptrs), std::end(ptrs), net.fwdPtrs);
    ck(cudaEventRecord(net.ev0, st), "cudaEventRecord");
    if (replay) ck(cudaGraphLaunch(net.fwdExec, st), "cudaGraphLaunch");
    else inferenceSequence(dRad, dFeat, N, H, W, Hp, Wp, dOut, st);
    ck(cudaGetLastError(), "denoiser launch");
    ck(cudaEventRecord(net.ev1, st), "cudaEventRecord");
    if (!replay) {   // capture after the timing event, so that the host work of the capture is not timed
        // the eager run may have allocated buffers (generation bumped): the graph is keyed on the state after it
        const int afterKey[7] = {N, H, W, Hp, Wp, net.tcMode, static_cast<int>(net.allocGen)};
        const void* const after[7] = {dRad, dFeat, dOut, net.act[0].p, net.wk.p, net.w.p, net.rowScratch.p};
        captureInference(dRad, dFeat, N, H, W, Hp, Wp, dOut, afterKey, after);
    }
    ck(cudaEventSynchronize(net.ev1), "denoise");
    ck(cudaEventElapsedTime(&net.lastMs, net.ev0, net.ev1), "cudaEventElapsedTime");
    checkTcFlag();
}

bool denoiserReady()
{
    std::lock_guard<std::mutex> lk(netMutex);
    return net.ready;
}

void denoiseForRenderer(const float* dRad, const float* dFeat, int N, int H, int W, float* dOut, cudaStream_t waitOn)
{
    std::lock_guard<std::mutex> lk(netMutex);
    try {
        ensureNet();
        denoiseDevice(dRad, dFeat, N, H, W, dOut, waitOn);
    } catch (const CudaErr& e) {
        throw std::runtime_error(e.msg);
    }
}

}  // namespace dn
}  // namespace bte

using namespace bte::dn;

extern "C" {

int bte_denoiser_init(uint64_t seed)
{
    return guardedDn([&] { initParams(seed); return 0; });
}

int bte_denoiser_param_count(long long* count)
{
    return guardedDn([&] {
        ensureNet();
        if (count) *count = static_cast<long long>(net.paramCount);
        return 0;
    });
}

int bte_denoiser_get_params(float* host, long long count)
{
    return guardedDn([&] {
        if (!net.ready) throw CudaErr{"bte_denoiser_get_params: not initialised"};
        if (count != static_cast<long long>(net.paramCount)) throw CudaErr{"bte_denoiser_get_params: wrong count"};
        ck(cudaMemcpyAsync(host, net.w.p, net.paramCount * 4, cudaMemcpyDeviceToHost, net.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(net.stream), "sync");
        return 0;
    });
}

int bte_denoiser_set_params(const float* host, long long count)
{
    return guardedDn([&] {
        ensureNet();
        if (count != static_cast<long long>(net.paramCount)) throw CudaErr{"bte_denoiser_set_params: wrong count"};
        if (!net.ready) initParams(0);
        ck(cudaMemcpyAsync(net.w.p, host, net.paramCount * 4, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
        ck(cudaMemsetAsync(net.m.p, 0, net.paramCount * 4, net.stream), "cudaMemsetAsync");
        ck(cudaMemsetAsync(net.v.p, 0, net.paramCount * 4, net.stream), "cudaMemsetAsync");
        refreshCopies();
        ck(cudaStreamSynchronize(net.stream), "sync");
        net.adamStep = 0;
        return 0;
    });
}

int bte_denoiser_set_dataset(const float* noisy, const float* features, const float* target, int count, int width,
                             int height)
{
    return guardedDn([&] {
        ensureNet();
        if (count <= 0 || width <= 0 || height <= 0 || !noisy || !features || !target)
            throw CudaErr{"bte_denoiser_set_dataset: empty set"};
        const size_t px = static_cast<size_t>(count) * width * height;
        net.dsNoisy.ensure(px * 12);
        net.dsFeat.ensure(px * 24);
        net.dsTarget.ensure(px * 12);
        ck(cudaMemcpyAsync(net.dsNoisy.p, noisy, px * 12, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(net.dsFeat.p, features, px * 24, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(net.dsTarget.p, target, px * 12, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(net.stream), "sync");
        net.dsCount = count; net.dsW = width; net.dsH = height;
        return 0;
    });
}

// `steps` Adam steps on batches of `batch` random crops (crop x crop, a
// multiple of 16, flipped at random); lossPerStep[steps] receives the mean
// L1 (log space) of each step.
int bte_denoiser_train(int steps, int batch, int crop, float learningRate, uint64_t seed, float* lossPerStep)
{
    return guardedDn([&] {
        if (!net.ready) throw CudaErr{"bte_denoiser_train: not initialised (bte_denoiser_init)"};
        if (net.dsCount <= 0) throw CudaErr{"bte_denoiser_train: no training set (bte_denoiser_set_dataset)"};
        if (steps <= 0 || batch <= 0 || crop <= 0 || crop % kAlign != 0 || crop > net.dsW || crop > net.dsH)
            throw CudaErr{"bte_denoiser_train: crop must be a positive multiple of 16 within the images"};
        cudaStream_t st = net.stream;
        ensureActs(batch, crop, crop, true);
        const size_t px = static_cast<size_t>(batch) * crop * crop;
        net.rad.ensure(px * 12);
        net.feat.ensure(px * 24);
        net.target.ensure(px * 12);
        net.lossSum.ensure(sizeof(float) * steps);
        net.params.ensure(sizeof(int) * 4 * batch * steps);
        std::mt19937_64 rng(seed);
        std::vector<int> hp(static_cast<size_t>(4) * batch * steps);
        for (int s = 0; s < steps; ++s)
            for (int b = 0; b < batch; ++b) {
                int* q = &hp[(static_cast<size_t>(s) * batch + b) * 4];
                q[0] = static_cast<int>(rng() % static_cast<uint64_t>(net.dsCount));
                q[1] = static_cast<int>(rng() % static_cast<uint64_t>(net.dsW - crop + 1));
                q[2] = static_cast<int>(rng() % static_cast<uint64_t>(net.dsH - crop + 1));
                q[3] = static_cast<int>(rng() & 3u);
            }
        ck(cudaMemcpyAsync(net.params.p, hp.data(), hp.size() * sizeof(int), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        ck(cudaMemsetAsync(net.lossSum.p, 0, sizeof(float) * steps, st), "cudaMemsetAsync");
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        ck(cudaEventRecord(net.ev0, st), "cudaEventRecord");
        for (int s = 0; s < steps; ++s) {
            gatherBatch(net.dsNoisy.as<float>(), net.dsFeat.as<float>(), net.dsTarget.as<float>(), net.dsW, net.dsH,
                        net.params.as<int>() + static_cast<size_t>(4) * batch * s, batch, crop, net.rad.as<float>(),
                        net.feat.as<float>(), net.target.as<float>(), st);
            assemble(net.rad.as<float>(), net.feat.as<float>(), batch, crop, crop, crop, crop, net.act[0].p, st);
            forward(batch, crop, crop, true);
            lossL1(net.act[27].p, net.act[0].p, net.target.as<float>(), static_cast<long long>(px), net.gact[27].p,
                   net.lossSum.as<float>() + s, st);
            backward(batch, crop, crop);
            ++net.adamStep;
            const float c1 = 1.0f - static_cast<float>(std::pow(b1, static_cast<double>(net.adamStep)));
            const float c2 = 1.0f - static_cast<float>(std::pow(b2, static_cast<double>(net.adamStep)));
            adam(net.w.as<float>(), net.grad.as<float>(), net.m.as<float>(), net.v.as<float>(),
                 static_cast<long long>(net.paramCount), learningRate, b1, b2, eps, c1, c2, st);
            refreshCopies();
        }
        ck(cudaGetLastError(), "training launch");
        ck(cudaEventRecord(net.ev1, st), "cudaEventRecord");
        std::vector<float> sums(static_cast<size_t>(steps));
        ck(cudaMemcpyAsync(sums.data(), net.lossSum.p, sizeof(float) * steps, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(st), "train");
        ck(cudaEventElapsedTime(&net.lastMs, net.ev0, net.ev1), "cudaEventElapsedTime");
        checkTcFlag();
        if (lossPerStep)
            for (int s = 0; s < steps; ++s) lossPerStep[s] = sums[static_cast<size_t>(s)] / static_cast<float>(px * 3);
        return 0;
    });
}

// Host radiance [H][W][3] and features [H][W][6] (may be null) -> host [H][W][3].
int bte_denoiser_denoise(const float* radiance, const float* features, int width, int height, float* out)
{
    return guardedDn([&] {
        ensureNet();
        if (width <= 0 || height <= 0 || !radiance || !out) throw CudaErr{"bte_denoiser_denoise: bad arguments"};
        const size_t px = static_cast<size_t>(width) * height;
        net.rad.ensure(px * 12);
        net.feat.ensure(px * 24);
        net.out.ensure(px * 12);
        ck(cudaMemcpyAsync(net.rad.p, radiance, px * 12, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
        if (features)
            ck(cudaMemcpyAsync(net.feat.p, features, px * 24, cudaMemcpyHostToDevice, net.stream), "cudaMemcpyAsync");
        denoiseDevice(net.rad.as<float>(), features ? net.feat.as<float>() : nullptr, 1, height, width, net.out.as<float>(),
                      nullptr);
        ck(cudaMemcpyAsync(out, net.out.p, px * 12, cudaMemcpyDeviceToHost, net.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(net.stream), "sync");
        return 0;
    });
}

// convolution kernels: 0 the warp-level mma.sync kernel only; 1 tcgen05 pixel tiles; 2 tcgen05 row tiles (decoder
// inputs upsampled first); 3 tcgen05 row tiles expanding upsampled inputs in shared memory
int bte_denoiser_set_tcgen05(int mode)
{
    return guardedDn([&] {
        if (mode < 0 || mode > 3) throw CudaErr{"bte_denoiser_set_tcgen05: mode must be 0, 1, 2 or 3"};
        ensureNet();
        net.tcMode = mode;
        return 0;
    });
}

// The failure path of the tensor-core kernels' pipeline waits, exercised without a fault: a wait on a barrier
// that nothing completes gives up after about two seconds; the status and duration come back to the host and
// the context stays usable.
int bte_denoiser_debug_wait_timeout(unsigned int* status, double* seconds)
{
    return guardedDn([&] {
        ensureNet();
        Buf b;
        b.ensure(16);
        ck(cudaMemsetAsync(b.p, 0, 16, net.stream), "cudaMemsetAsync");
        waitTimeoutProbe(b.as<unsigned int>(), reinterpret_cast<unsigned long long*>(b.as<unsigned char>() + 8),
                         net.stream);
        ck(cudaGetLastError(), "probe launch");
        unsigned char host[16];
        ck(cudaMemcpyAsync(host, b.p, 16, cudaMemcpyDeviceToHost, net.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(net.stream), "sync");
        b.release();
        unsigned int st = 0;
        unsigned long long ns = 0;
        std::memcpy(&st, host, 4);
        std::memcpy(&ns, host + 8, 8);
        if (status) *status = st;
        if (seconds) *seconds = static_cast<double>(ns) * 1e-9;
        return 0;
    });
}

// weight-gradient kernel of training: 1 (default) the tcgen05 kernel for the layers whose shapes it takes (image
// width a multiple of 8, pixels a multiple of 64), the warp-level one for the rest; 0 the warp-level mma.sync kernel;
// 2 to 1 + kWgradTcVariants: the tcgen05 kernel with pipeline shape kind - 1 (a tuning choice; the sums are the same)
int bte_denoiser_set_wgrad(int kind)
{
    return guardedDn([&] {
        if (kind < 0 || kind > 1 + kWgradTcVariants)
            throw CudaErr{"bte_denoiser_set_wgrad: kind must be 0 (warp-level), 1 (tcgen05) or 2 to " +
                          std::to_string(1 + kWgradTcVariants) + " (tcgen05 pipeline shapes)"};
        ensureNet();
        net.wgradKind = kind;
        return 0;
    });
}

int bte_denoiser_last_ms(float* ms)
{
    return guardedDn([&] {
        if (ms) *ms = net.lastMs;
        return 0;
    });
}

// Kernel-level entry for numerical checks: op 0 forward conv (x, w, bias ->
// out [N,H,W,Cout]), op 1 data gradient (dy, w -> out [N,H,W,Cin]), op 2 weight
// gradient (x, dy -> out [9][Cout][Cin] followed by [Cout] bias gradient); ops 3, 4
// and 5, 6 are ops 0, 1 on the tcgen05 pixel-tile and row-tile kernels.
// Host FP32 arrays are rounded to bf16 on the device; w is [9][Cout][Cin].
int bte_denoiser_debug_conv(int op, const float* x, const float* w, const float* bias, const float* dy, int n, int h,
                            int wd, int cin, int cout, int relu, float* out)
{
    return guardedDn([&] {
        ensureNet();
        if (cin % 16 || cout % 16 || n <= 0 || h <= 0 || wd <= 0) throw CudaErr{"bte_denoiser_debug_conv: bad shape"};
        cudaStream_t st = net.stream;
        const size_t px = static_cast<size_t>(n) * h * wd;
        Buf bx, bb, bdy, bo, bf32, bwk, bwd;
        // float -> bf16 through the weight-copy kernel, viewing the array as [9 taps][1][count/9]
        auto convert = [&](const float* host, size_t count, Buf& dst) {
            const size_t padded = (count + 8) / 9 * 9;
            std::vector<float> tmp(padded, 0.0f);
            std::memcpy(tmp.data(), host, count * 4);
            bf32.ensure(padded * 4);
            dst.ensure(padded * 2);
            ck(cudaMemcpyAsync(bf32.p, tmp.data(), padded * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
            weightCopies(bf32.as<float>(), static_cast<int>(padded / 9), 1, dst.p, nullptr, st);
            ck(cudaStreamSynchronize(st), "sync");
        };
        if (op < 0 || op > 7) throw CudaErr{"bte_denoiser_debug_conv: op must be 0 to 7"};
        const bool wgradTc = op == 7;
        if (wgradTc) {
            if (!convWgradTcSupported(n, h, wd, cin, cout))
                throw CudaErr{"bte_denoiser_debug_conv: shape not supported by the tcgen05 weight gradient"};
            op = 2;
        }
        // ops 3 and 4: ops 0 and 1 on the tcgen05 pixel-tile kernel; ops 5 and 6 on the row-tile kernel
        const int force = op >= 5 ? 2 : (op >= 3 ? 1 : 0);
        if (op >= 5) op -= 5;
        else if (op >= 3) op -= 3;
        if (op == 0 || op == 1) {
            const int inC = op == 0 ? cin : cout, outC = op == 0 ? cout : cin;
            convert(op == 0 ? x : dy, px * inC, bx);
            // weights: forward copy and data-gradient copy from FP32 [9][cout][cin]
            Buf wf;
            wf.ensure(9ull * cin * cout * 4);
            ck(cudaMemcpyAsync(wf.p, w, 9ull * cin * cout * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
            bwk.ensure(9ull * cin * cout * 2);
            bwd.ensure(9ull * cin * cout * 2);
            weightCopies(wf.as<float>(), cin, cout, bwk.p, bwd.p, st);
            if (op == 0 && bias) {
                bb.ensure(cout * 4ull);
                ck(cudaMemcpyAsync(bb.p, bias, cout * 4ull, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
            }
            bo.ensure(px * outC * 2);
            convDispatch(bx.p, inC, false, nullptr, 0, n, h, wd, op == 0 ? bwk.p : bwd.p,
                         op == 0 && bias ? bb.as<float>() : nullptr, outC, op == 0 && relu, bo.p, st, force);
            ck(cudaGetLastError(), "conv launch");
            checkTcFlag();
            // bf16 -> float on the host
            std::vector<unsigned short> hb(px * outC);
            ck(cudaMemcpyAsync(hb.data(), bo.p, hb.size() * 2, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
            ck(cudaStreamSynchronize(st), "sync");
            for (size_t i = 0; i < hb.size(); ++i) {
                const uint32_t u = static_cast<uint32_t>(hb[i]) << 16;
                std::memcpy(out + i, &u, 4);
            }
            wf.release();
        } else if (op == 2) {
            convert(x, px * cin, bx);
            convert(dy, px * cout, bdy);
            Buf g;
            g.ensure((9ull * cin * cout + cout) * 4);
            ck(cudaMemsetAsync(g.p, 0, (9ull * cin * cout + cout) * 4, st), "cudaMemsetAsync");
            Buf scratch;
            if (wgradTc) {
                scratch.ensure(convWgradTcScratchBytes(n, h, wd, cin, cout));
                convWgradTc(bx.p, bdy.p, n, h, wd, cin, cout, g.as<float>(), scratch.p, net.errFlag.as<unsigned int>(), st,
                            net.wgradKind >= 2 ? net.wgradKind - 1 : 0);
            } else {
                convWgrad(bx.p, bdy.p, n, h, wd, cin, cout, g.as<float>(), st);
            }
            biasGrad(bdy.p, static_cast<long long>(px), cout, g.as<float>() + 9ull * cin * cout, st);
            ck(cudaGetLastError(), "wgrad launch");
            ck(cudaMemcpyAsync(out, g.p, (9ull * cin * cout + cout) * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
            ck(cudaStreamSynchronize(st), "sync");
            if (wgradTc) checkTcFlag();
            g.release();
            scratch.release();
        } else {
            throw CudaErr{"bte_denoiser_debug_conv: op must be 0 to 6"};
        }
        bx.release(); bb.release(); bdy.release(); bo.release(); bf32.release(); bwk.release(); bwd.release();
        return 0;
    });
}

}  // extern "C"
