// bte_denoise.h -- launchers of the denoiser kernels (bte_denoise_kernels.cu).
// Tensors are NHWC bf16 (passed as void*), channel counts multiples of 16.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace bte {
namespace dn {

// Y = act(conv3x3(X, Wk) + bias); Wk[9][Cout][Cin] bf16, zero padding at the borders.
void conv3x3(const void* X, int N, int H, int W, int Cin, const void* Wk, const float* bias, int Cout, bool relu, void* Y,
             cudaStream_t st);
// Same with the input concat(up ? nearest-upsample-2x(X1) : X1, X2) read in
// place (X1 has C1 channels, X2 has C2, Wk's Cin = C1 + C2).
void conv3x3Cat(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
                const float* bias, int Cout, bool relu, void* Y, cudaStream_t st);
// The same convolution on the tcgen05 tensor cores (accumulator in TMEM);
// sets *errorFlag on an internal timeout.  Cout: multiple of 16, <= 256.
bool convTcSupported(int Cin, int Cout);
void conv3x3Tc(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
               const float* bias, int Cout, bool relu, void* Y, unsigned int* errorFlag, cudaStream_t st);
// The row-tile tcgen05 kernel: 128-pixel row segments, the 3-row input slab
// staged once per tile (TMA), weights resident in shared memory, warp-
// specialised copy / MMA / epilogue.  Cout 16, 32, 48, 64, 96 or 128; C1 and C2
// multiples of 8 with Cin a multiple of 16.  A layer whose weights and slabs
// do not fit shared memory runs in passes over its input channels, summing in
// an FP32 scratch buffer of convTcRowScratchBytes (0 for a single pass).
bool convTcRowSupported(int C1, int C2, bool up, int Cout);
size_t convTcRowScratchBytes(int C1, int C2, bool up, int Cout, int N, int H, int W);
// pool (optional): also write the 2x2 average pool of Y there when the last pass runs two-row tiles;
// returns whether it did.
bool conv3x3TcRow(const void* X1, int C1, bool up, const void* X2, int C2, int N, int H, int W, const void* Wk,
                  const float* bias, int Cout, bool relu, void* Y, void* scratch, void* pool, unsigned int* errorFlag,
                  cudaStream_t st);
// Runs the tcgen05 kernels' bounded pipeline wait on an mbarrier that nothing completes (one warp):
// *dStatus 2 when the wait gave up, 1 if it returned as completed; *dNs its duration.
void waitTimeoutProbe(unsigned int* dStatus, unsigned long long* dNs, cudaStream_t st);
// The weight gradient on the tcgen05 tensor cores (pixels as the reduction axis, channel-major copies of dY and
// of the column-shifted X made first in `scratch`, convWgradTcScratchBytes of it); same sums as convWgrad.
// Needs W % 8 == 0, N*H*W % 64 == 0, 16 <= Cin <= 256, Cout <= 128; sets *errorFlag on an internal timeout.
bool convWgradTcSupported(int N, int H, int W, int Cin, int Cout);
size_t convWgradTcScratchBytes(int N, int H, int W, int Cin, int Cout);
// `variant` picks the pipeline shape (stages, copy lag, pixels per stage): 1 (3, 2, 64), 2 (4, 2, 64), 3 (6, 4, 32),
// 4 (5, 3, 32) with zero-filling copies; 5 (3, 2, 64) and 6 (5, 3, 32) with plain copies of the in-range chunks and
// shared-memory zero stores for the rest; 0 the default, kWgradTcDefaultVariant.
constexpr int kWgradTcDefaultVariant = 1;
constexpr int kWgradTcVariants = 6;
void convWgradTc(const void* X, const void* dY, int N, int H, int W, int Cin, int Cout, float* dW, void* scratch,
                 unsigned int* errorFlag, cudaStream_t st, int variant = 0);
// dW[9][Cout][Cin] += sum over pixels of dY x shifted X (FP32 atomics).
void convWgrad(const void* X, const void* dY, int N, int H, int W, int Cin, int Cout, float* dW, cudaStream_t st);
void biasGrad(const void* dY, long long pixels, int C, float* db, cudaStream_t st);
void reluMask(const void* Y, const void* dY, void* out, long long elems, cudaStream_t st);
void pool2(const void* X, int N, int H, int W, int C, void* Y, cudaStream_t st);
void pool2Back(const void* dY, int N, int H, int W, int C, void* dX, cudaStream_t st);   // adds into dX
void upCat(const void* A, int Ca, const void* B, int Cb, int N, int H, int W, void* out, cudaStream_t st);
// nearest 2x upsampling of X [N][Hs][Ws][C] (C a multiple of 8) into Y [N][2Hs][2Ws][C]
void upsample2(const void* X, int N, int Hs, int Ws, int C, void* Y, cudaStream_t st);
void upCatBack(const void* dOut, int Ca, int Cb, int N, int H, int W, void* dA, void* dB, bool addB, cudaStream_t st);
void assemble(const float* rad, const float* feat, int N, int H, int W, int Hp, int Wp, void* out, cudaStream_t st);
void output(const void* net, const void* in, int N, int H, int W, int Hp, int Wp, float* rad, cudaStream_t st);
void lossL1(const void* net, const void* in, const float* target, long long pixels, void* dNet, float* lossSum,
            cudaStream_t st);
void adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps, float c1,
          float c2, cudaStream_t st);
void weightCopies(const float* w, int Cin, int Cout, void* wk, void* wd, cudaStream_t st);
// batch of crops from a device-resident set of images (training)
void gatherBatch(const float* noisy, const float* feat, const float* target, int width, int height, const int* params,
                 int batch, int crop, float* bRad, float* bFeat, float* bTarget, cudaStream_t st);

// Denoise the renderer's accumulation: dRad [N][H][W][3] mean radiance,
// dFeat [N][H][W][6] (or null) -> dOut [N][H][W][3]; waits for `waitOn`
// first and returns when done.  Throws std::runtime_error.
void denoiseForRenderer(const float* dRad, const float* dFeat, int N, int H, int W, float* dOut, cudaStream_t waitOn);
bool denoiserReady();

}  // namespace dn
}  // namespace bte
