// bte_bvh.cu -- LBVH construction on the GPU (replaces the OptiX GAS build,
// src/host/optix_setup.cu:215-292).
//
//   1. per-triangle bounds and centroids; scene centroid bounds (order-free
//      min/max reduction through monotone integer encodings)
//   2. 63-bit Morton codes (21 bits per axis)
//   3. stable LSD radix sort of (code, triangle) pairs, 4-bit digits
//      (16 passes); ties keep ascending triangle order
//   4. hierarchy from the sorted codes (T. Karras, "Maximizing Parallelism in
//      the Construction of BVHs, Octrees, and k-d Trees", HPG 2012), equal
//      codes separated by their index
//   5. bottom-up refit with one atomic arrival counter per node, with a
//      surface-area cost decision collapsing small subtrees (contiguous
//      ranges of the sorted triangles) into multi-triangle leaves
//   6. output: 64-byte BVH2 nodes holding both child boxes, or an 8-wide tree
//      of 80-byte nodes with quantised boxes collapsed from the binary one,
//      and the triangles in leaf order as three float4 each (v0|original
//      index, v1, v2)
// All integer steps are deterministic; the result does not depend on thread
// scheduling.
#include "bte_kernels.h"

#include <cfloat>
#include <climits>
#include <vector>

namespace bte {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kDigits = 16;

__device__ __forceinline__ unsigned int floatToOrdered(float f)
{
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedToFloat(unsigned int u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void kTriPrep(const TriangleData* __restrict__ tris, int n, float4* cen, unsigned int* bounds)
{
    __shared__ unsigned int sLo[3], sHi[3];
    if (threadIdx.x < 3) { sLo[threadIdx.x] = 0xffffffffu; sHi[threadIdx.x] = 0u; }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const TriangleData t = tris[i];
        const float lx = fminf(t.v0.x, fminf(t.v1.x, t.v2.x)), hx = fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x));
        const float ly = fminf(t.v0.y, fminf(t.v1.y, t.v2.y)), hy = fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y));
        const float lz = fminf(t.v0.z, fminf(t.v1.z, t.v2.z)), hz = fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z));
        const float cx = 0.5f * (lx + hx), cy = 0.5f * (ly + hy), cz = 0.5f * (lz + hz);
        cen[i] = make_float4(cx, cy, cz, 0.0f);
        atomicMin(&sLo[0], floatToOrdered(cx)); atomicMax(&sHi[0], floatToOrdered(cx));
        atomicMin(&sLo[1], floatToOrdered(cy)); atomicMax(&sHi[1], floatToOrdered(cy));
        atomicMin(&sLo[2], floatToOrdered(cz)); atomicMax(&sHi[2], floatToOrdered(cz));
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&bounds[threadIdx.x], sLo[threadIdx.x]);
        atomicMax(&bounds[3 + threadIdx.x], sHi[threadIdx.x]);
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned int v)
{
    unsigned long long x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

__global__ void kMorton(const float4* __restrict__ cen, int n, const unsigned int* bounds, unsigned long long* keys,
                        int* vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lo[3] = {orderedToFloat(bounds[0]), orderedToFloat(bounds[1]), orderedToFloat(bounds[2])};
    const float hi[3] = {orderedToFloat(bounds[3]), orderedToFloat(bounds[4]), orderedToFloat(bounds[5])};
    const float4 c = cen[i];
    const float cc[3] = {c.x, c.y, c.z};
    unsigned int q[3];
    for (int k = 0; k < 3; ++k) {
        const float ext = hi[k] - lo[k];
        float f = (ext > 0.0f) ? (cc[k] - lo[k]) / ext : 0.0f;
        f = fminf(fmaxf(f, 0.0f), 1.0f);
        q[k] = min(static_cast<unsigned int>(f * 2097152.0f), 2097151u);
    }
    keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    vals[i] = i;
}

__global__ void kRadixHist(const unsigned long long* __restrict__ keys, int n, int shift, int numTiles, int* hist)
{
    __shared__ int cnt[kDigits];
    if (threadIdx.x < kDigits) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    for (int j = 0; j < kSortItems; ++j) {
        const int i = base + j * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[static_cast<int>((keys[i] >> shift) & 0xf)], 1);
    }
    __syncthreads();
    if (threadIdx.x < kDigits) hist[threadIdx.x * numTiles + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of hist[0..m) by one block
__global__ void kScanSingle(int* data, int m)
{
    __shared__ int carry;
    __shared__ int warpSums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < m; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = (i < m) ? data[i] : 0;
        int x = v;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = (lane < static_cast<int>(blockDim.x >> 5)) ? warpSums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warpSums[lane] = w;
        }
        __syncthreads();
        const int warpPrefix = (warp > 0) ? warpSums[warp - 1] : 0;
        const int incl = x + warpPrefix;
        if (i < m) data[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
}

// Stable scatter: element order within a tile is thread-major (thread t owns
// items t*kSortItems .. +kSortItems-1 of the tile).
__global__ void kRadixScatter(const unsigned long long* __restrict__ keysIn, const int* __restrict__ valsIn,
                              unsigned long long* keysOut, int* valsOut, int n, int shift, int numTiles,
                              const int* __restrict__ histScan)
{
    __shared__ int cnt[kDigits][kSortThreads + 1];
    __shared__ int gbase[kDigits];
    const int t = threadIdx.x;
    const int tileBase = blockIdx.x * kSortTile + t * kSortItems;
    unsigned long long k[kSortItems];
    int v[kSortItems];
    int dg[kSortItems];
    for (int d = 0; d < kDigits; ++d) cnt[d][t] = 0;
    for (int j = 0; j < kSortItems; ++j) {
        const int i = tileBase + j;
        if (i < n) {
            k[j] = keysIn[i];
            v[j] = valsIn[i];
            dg[j] = static_cast<int>((k[j] >> shift) & 0xf);
        } else {
            dg[j] = -1;
        }
    }
    for (int j = 0; j < kSortItems; ++j) if (dg[j] >= 0) cnt[dg[j]][t] += 1;
    if (t < kDigits) gbase[t] = histScan[t * numTiles + blockIdx.x];
    __syncthreads();
    if (t < kDigits) {   // exclusive scan over threads for digit t
        int run = 0;
        for (int u = 0; u < kSortThreads; ++u) {
            const int c = cnt[t][u];
            cnt[t][u] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int j = 0; j < kSortItems; ++j) {
        if (dg[j] < 0) continue;
        int rank = 0;
        for (int jj = 0; jj < j; ++jj) rank += (dg[jj] == dg[j]) ? 1 : 0;
        const int pos = gbase[dg[j]] + cnt[dg[j]][t] + rank;
        keysOut[pos] = k[j];
        valsOut[pos] = v[j];
    }
}

__device__ __forceinline__ int delta(const unsigned long long* keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const unsigned long long a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(static_cast<unsigned int>(i) ^ static_cast<unsigned int>(j));
    return __clzll(a ^ b);
}

// internal node i in [0, n-2]; children encoded >= 0 internal, < 0 leaf ~k
__global__ void kKarras(const unsigned long long* __restrict__ keys, int n, int2* children, int* parentInner,
                        int* parentLeaf, int2* range)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int s = 0;
    int div = 2;
    int t;
    do {
        t = (l + div - 1) / div;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        div *= 2;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    int left, right;
    if (lo == gamma) { left = ~gamma; parentLeaf[gamma] = i; }
    else { left = gamma; parentInner[gamma] = i; }
    if (hi == gamma + 1) { right = ~(gamma + 1); parentLeaf[gamma + 1] = i; }
    else { right = gamma + 1; parentInner[gamma + 1] = i; }
    children[i] = make_int2(left, right);
    range[i] = make_int2(lo, hi);
    if (i == 0) parentInner[0] = -1;
}

struct Box { float lx, ly, lz, hx, hy, hz; };

__device__ __forceinline__ Box triBox(const TriangleData& t)
{
    Box b;
    b.lx = fminf(t.v0.x, fminf(t.v1.x, t.v2.x)); b.hx = fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x));
    b.ly = fminf(t.v0.y, fminf(t.v1.y, t.v2.y)); b.hy = fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y));
    b.lz = fminf(t.v0.z, fminf(t.v1.z, t.v2.z)); b.hz = fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z));
    return b;
}

// leaf k (sorted position) -> leaf triangle data + its box; walks up and
// fills the inner nodes' boxes (second arrival computes the union).
// Surface-area cost model for collapsing subtrees into leaves: a node becomes
// a leaf of its whole (contiguous) triangle range when that is no costlier
// than keeping the split (kCostTrav per node visit, kCostIsect per triangle).
constexpr float kCostTrav = 1.2f;
constexpr float kCostIsect = 1.0f;

__device__ __forceinline__ float halfArea(const float* b)
{
    const float dx = fmaxf(b[3] - b[0], 0.0f), dy = fmaxf(b[4] - b[1], 0.0f), dz = fmaxf(b[5] - b[2], 0.0f);
    return dx * dy + dy * dz + dz * dx;
}

__global__ void kRefit(const TriangleData* __restrict__ tris, const int* __restrict__ sortedTri, int n,
                       const int2* __restrict__ children, const int* __restrict__ parentInner,
                       const int* __restrict__ parentLeaf, const int2* __restrict__ range, float4* leafTris,
                       float* innerBox /*[n-1][6]*/, float* leafBox /*[n][6]*/, int* arrivals, float* cost,
                       int* collapsed, int maxLeaf)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int ti = sortedTri[k];
    const TriangleData t = tris[ti];
    leafTris[3 * k] = make_float4(t.v0.x, t.v0.y, t.v0.z, __int_as_float(ti));
    leafTris[3 * k + 1] = make_float4(t.v1.x, t.v1.y, t.v1.z, 0.0f);
    leafTris[3 * k + 2] = make_float4(t.v2.x, t.v2.y, t.v2.z, 0.0f);
    const Box b = triBox(t);
    float* lb = leafBox + 6 * static_cast<size_t>(k);
    lb[0] = b.lx; lb[1] = b.ly; lb[2] = b.lz; lb[3] = b.hx; lb[4] = b.hy; lb[5] = b.hz;
    if (n < 2) return;
    __threadfence();
    int node = parentLeaf[k];
    while (node >= 0) {
        if (atomicAdd(&arrivals[node], 1) == 0) return;   // first arrival: sibling not ready
        __threadfence();
        const int2 c = children[node];
        float a[6], bb[6];
        const float* pa = (c.x >= 0) ? innerBox + 6 * static_cast<size_t>(c.x) : leafBox + 6 * static_cast<size_t>(~c.x);
        const float* pb = (c.y >= 0) ? innerBox + 6 * static_cast<size_t>(c.y) : leafBox + 6 * static_cast<size_t>(~c.y);
        for (int q = 0; q < 6; ++q) { a[q] = __ldcg(pa + q); bb[q] = __ldcg(pb + q); }
        float* out = innerBox + 6 * static_cast<size_t>(node);
        float u[6];
        u[0] = fminf(a[0], bb[0]); u[1] = fminf(a[1], bb[1]); u[2] = fminf(a[2], bb[2]);
        u[3] = fmaxf(a[3], bb[3]); u[4] = fmaxf(a[4], bb[4]); u[5] = fmaxf(a[5], bb[5]);
        for (int q = 0; q < 6; ++q) out[q] = u[q];
        const float cl = (c.x >= 0) ? __ldcg(cost + c.x) : kCostIsect;
        const float cr = (c.y >= 0) ? __ldcg(cost + c.y) : kCostIsect;
        const float A = halfArea(u);
        const float split = (A > 0.0f) ? kCostTrav + (halfArea(a) * cl + halfArea(bb) * cr) / A : kCostTrav + cl + cr;
        const int2 rg = range[node];
        const int cnt = rg.y - rg.x + 1;
        const float leafCost = kCostIsect * static_cast<float>(cnt);
        const bool col = cnt <= maxLeaf && leafCost <= split;
        cost[node] = col ? leafCost : split;
        collapsed[node] = col ? 1 : 0;
        __threadfence();
        node = parentInner[node];
    }
}

__device__ __forceinline__ int leafCode(int start, int count) { return ~(start | ((count - 1) << kLeafCountShift)); }

__global__ void kEmitNodes(const int2* __restrict__ children, const float* __restrict__ innerBox,
                           const float* __restrict__ leafBox, const int2* __restrict__ range,
                           const int* __restrict__ collapsed, int n, BvhNode* nodes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int2 c = children[i];
    const float* a = (c.x >= 0) ? innerBox + 6 * static_cast<size_t>(c.x) : leafBox + 6 * static_cast<size_t>(~c.x);
    const float* b = (c.y >= 0) ? innerBox + 6 * static_cast<size_t>(c.y) : leafBox + 6 * static_cast<size_t>(~c.y);
    BvhNode nd;
    nd.lxy = make_float4(a[0], a[3], a[1], a[4]);
    nd.rxy = make_float4(b[0], b[3], b[1], b[4]);
    nd.z = make_float4(a[2], a[5], b[2], b[5]);
    int e0 = c.x, e1 = c.y;   // ~k is already the leaf code of a single triangle
    if (c.x >= 0 && collapsed[c.x]) e0 = leafCode(range[c.x].x, range[c.x].y - range[c.x].x + 1);
    if (c.y >= 0 && collapsed[c.y]) e1 = leafCode(range[c.y].x, range[c.y].y - range[c.y].x + 1);
    nd.child = make_int4(e0, e1, 0, 0);
    nodes[i] = nd;
}

// ---------------------------------------------------------------- PLOC
// Parallel locally-ordered clustering (D. Meister, J. Bittner, "Parallel
// Locally-Ordered Clustering for Bounding Volume Hierarchy Construction",
// IEEE TVCG 24(3), 2018), the alternative to the Morton-prefix hierarchy.
// Clusters start as the triangles in Morton order.  Each round every cluster
// picks, among the clusters at most `radius` positions away, the one whose
// union box has the smallest surface area, ties going to the lower position.
// That makes the choice the minimum of a strict total order over pairs
// (area, lower position, higher position), so the best pair of the round is
// always mutual and every round merges.  Mutual pairs merge into a new inner
// node at the lower position; survivors are compacted in order.  Inner node
// ids are handed out downwards from n-2, so the last merge is the root 0.
// The tree is then relabelled in depth-first order (subtree triangle counts,
// first-leaf offsets) so that every subtree is a contiguous range of leaves,
// which is what the refit, the leaf collapse and the 8-wide collapse expect.
constexpr int kPlocBlock = 256;
constexpr int kPlocItems = 4;
constexpr int kPlocTile = kPlocBlock * kPlocItems;

struct Cluster {
    float4 lo;   // box min, w: node code (>= 0 inner node, ~k Morton-order triangle k)
    float4 hi;   // box max, w: triangles below
};

__global__ void kPlocInit(const TriangleData* __restrict__ tris, const int* __restrict__ sortedTri, int n, Cluster* c)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const Box b = triBox(tris[sortedTri[k]]);
    c[k].lo = make_float4(b.lx, b.ly, b.lz, __int_as_float(~k));
    c[k].hi = make_float4(b.hx, b.hy, b.hz, __int_as_float(1));
}

__device__ __forceinline__ float unionArea(const float4& alo, const float4& ahi, const float4& blo, const float4& bhi)
{
    const float dx = fmaxf(fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x), 0.0f);
    const float dy = fmaxf(fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y), 0.0f);
    const float dz = fmaxf(fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z), 0.0f);
    const float a = dx * dy + dy * dz + dz * dx;
    return (a == a) ? a : INFINITY;   // NaN coordinates: the farthest, still ordered by position
}

// nn[i] = the chosen neighbour of cluster i (-1 only when m == 1)
__global__ void __launch_bounds__(kPlocBlock) kPlocNearest(const Cluster* __restrict__ c, int m, int radius, int* nn)
{
    __shared__ float4 sLo[kPlocBlock + 2 * kPlocMaxRadius], sHi[kPlocBlock + 2 * kPlocMaxRadius];
    const int start = blockIdx.x * kPlocBlock - radius;
    for (int t = threadIdx.x; t < kPlocBlock + 2 * radius; t += kPlocBlock) {
        const int j = start + t;
        if (j >= 0 && j < m) { sLo[t] = c[j].lo; sHi[t] = c[j].hi; }
    }
    __syncthreads();
    const int i = blockIdx.x * kPlocBlock + threadIdx.x;
    if (i >= m) return;
    const float4 alo = sLo[i - start], ahi = sHi[i - start];
    const int jlo = max(0, i - radius), jhi = min(m - 1, i + radius);
    float best = INFINITY;
    int bestJ = -1;
    for (int j = jlo; j <= jhi; ++j) {
        if (j == i) continue;
        const float a = unionArea(alo, ahi, sLo[j - start], sHi[j - start]);
        if (bestJ < 0 || a < best) { best = a; bestJ = j; }   // ascending j: ties keep the lower position
    }
    nn[i] = bestJ;
}

// (survives, owns a merge) of cluster i
__device__ __forceinline__ int2 plocFlags(const int* __restrict__ nn, int m, int i)
{
    if (i >= m) return make_int2(0, 0);
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    return make_int2((mutual && i > j) ? 0 : 1, (mutual && i < j) ? 1 : 0);
}

__global__ void __launch_bounds__(kPlocBlock) kPlocCount(const int* __restrict__ nn, int m, int2* tileSums)
{
    __shared__ int2 warpSums[kPlocBlock / 32];
    const int base = blockIdx.x * kPlocTile;
    int2 s = make_int2(0, 0);
    for (int q = 0; q < kPlocItems; ++q) {
        const int2 f = plocFlags(nn, m, base + q * kPlocBlock + threadIdx.x);
        s.x += f.x; s.y += f.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_down_sync(0xffffffffu, s.x, o);
        s.y += __shfl_down_sync(0xffffffffu, s.y, o);
    }
    if ((threadIdx.x & 31) == 0) warpSums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int2 t = make_int2(0, 0);
        for (int w = 0; w < kPlocBlock / 32; ++w) { t.x += warpSums[w].x; t.y += warpSums[w].y; }
        tileSums[blockIdx.x] = t;
    }
}

// exclusive scan of tileSums[0..tiles) by one block of 1024 threads;
// tileSums[tiles] = totals
__global__ void __launch_bounds__(1024) kPlocScanTiles(int2* tileSums, int tiles)
{
    __shared__ int2 warpSums[32];
    __shared__ int2 carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = make_int2(0, 0);
    __syncthreads();
    for (int base = 0; base < tiles; base += 1024) {
        const int i = base + threadIdx.x;
        const int2 v = (i < tiles) ? tileSums[i] : make_int2(0, 0);
        int2 x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int yx = __shfl_up_sync(0xffffffffu, x.x, o), yy = __shfl_up_sync(0xffffffffu, x.y, o);
            if (lane >= o) { x.x += yx; x.y += yy; }
        }
        if (lane == 31) warpSums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int2 w = warpSums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int yx = __shfl_up_sync(0xffffffffu, w.x, o), yy = __shfl_up_sync(0xffffffffu, w.y, o);
                if (lane >= o) { w.x += yx; w.y += yy; }
            }
            warpSums[lane] = w;
        }
        __syncthreads();
        const int2 wp = (warp > 0) ? warpSums[warp - 1] : make_int2(0, 0);
        const int2 incl = make_int2(x.x + wp.x, x.y + wp.y);
        if (i < tiles) tileSums[i] = make_int2(carry.x + incl.x - v.x, carry.y + incl.y - v.y);
        __syncthreads();
        if (threadIdx.x == 1023) { carry.x += incl.x; carry.y += incl.y; }
        __syncthreads();
    }
    if (threadIdx.x == 0) tileSums[tiles] = carry;
}

// Survivors to their compacted position; each mutual pair's lower member
// becomes the new inner node `nextId - (merges before it)`.
__global__ void __launch_bounds__(kPlocBlock) kPlocCompact(const Cluster* __restrict__ c, const int* __restrict__ nn,
                                                           int m, const int2* __restrict__ tileScan, int nextId,
                                                           Cluster* out, int2* children, int* counts)
{
    __shared__ int2 warpSums[kPlocBlock / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int first = blockIdx.x * kPlocTile + t * kPlocItems;   // thread-major: keeps positions in order
    int2 f[kPlocItems];
    int2 s = make_int2(0, 0);
    for (int q = 0; q < kPlocItems; ++q) { f[q] = plocFlags(nn, m, first + q); s.x += f[q].x; s.y += f[q].y; }
    int2 x = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int yx = __shfl_up_sync(0xffffffffu, x.x, o), yy = __shfl_up_sync(0xffffffffu, x.y, o);
        if (lane >= o) { x.x += yx; x.y += yy; }
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    int2 pre = tileScan[blockIdx.x];
    for (int w = 0; w < warp; ++w) { pre.x += warpSums[w].x; pre.y += warpSums[w].y; }
    pre.x += x.x - s.x; pre.y += x.y - s.y;   // exclusive prefix of this thread's first item
    for (int q = 0; q < kPlocItems; ++q) {
        const int i = first + q;
        if (f[q].x) {
            Cluster a = c[i];
            if (f[q].y) {
                const Cluster b = c[nn[i]];
                const int id = nextId - pre.y;
                children[id] = make_int2(__float_as_int(a.lo.w), __float_as_int(b.lo.w));
                const int cnt = __float_as_int(a.hi.w) + __float_as_int(b.hi.w);
                counts[id] = cnt;
                a.lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), __int_as_float(id));
                a.hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), __int_as_float(cnt));
            }
            out[pre.x] = a;
        }
        pre.x += f[q].x; pre.y += f[q].y;
    }
}

__global__ void kPlocParents(const int2* __restrict__ children, int inner, int* parentInner, int* parentMorton)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= inner) return;
    const int2 c = children[id];
    if (c.x >= 0) parentInner[c.x] = id; else parentMorton[~c.x] = id;
    if (c.y >= 0) parentInner[c.y] = id; else parentMorton[~c.y] = id;
    if (id == 0) parentInner[0] = -1;
}

__device__ __forceinline__ int subtreeCount(const int* counts, int code) { return code >= 0 ? counts[code] : 1; }

// first leaf (depth-first order) of every inner node, by a walk to the root;
// depthMax = the deepest leaf's depth
__global__ void kPlocFirstInner(const int2* __restrict__ children, const int* __restrict__ parentInner,
                                const int* __restrict__ counts, int inner, int* firstInner, int* depthMax)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= inner) return;
    int first = 0, cur = id, depth = 1;
    for (int p = parentInner[cur]; p >= 0 && depth <= inner; cur = p, p = parentInner[p], ++depth) {
        const int2 c = children[p];
        if (c.y == cur) first += subtreeCount(counts, c.x);
    }
    firstInner[id] = first;
    atomicMax(depthMax, depth + 1);
}

// depth-first relabel: leaf codes, ranges, triangle order, leaf parents
__global__ void kPlocRelabel(int2* children, const int* __restrict__ counts, const int* __restrict__ firstInner,
                             const int* __restrict__ parentMorton, const int* __restrict__ sortedMorton, int n,
                             int2* range, int* sortedTri, int* parentLeaf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {   // leaf i in Morton order
        const int p = parentMorton[i];
        const int2 c = children[p];
        const int pos = firstInner[p] + ((c.y == ~i) ? subtreeCount(counts, c.x) : 0);
        sortedTri[pos] = sortedMorton[i];
        parentLeaf[pos] = p;
    }
    if (i < n - 1) {
        const int f = firstInner[i];
        range[i] = make_int2(f, f + counts[i] - 1);
    }
}

__global__ void kPlocLeafCodes(int2* children, const int* __restrict__ counts, const int* __restrict__ firstInner,
                               int inner)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= inner) return;
    int2 c = children[id];
    const int f = firstInner[id];
    if (c.x < 0) c.x = ~f;                               // the left child starts the parent's range
    if (c.y < 0) c.y = ~(f + subtreeCount(counts, c.x));
    children[id] = c;
}

// ---------------------------------------------------------------- 8-wide collapse
// Top-down, one level of the wide tree per pass.  A wide node rooted at a
// binary node takes its two children and then repeatedly opens the child of
// largest surface area that holds more than kWideLeafMax triangles (then, if
// slots remain, any child with two or more), up to eight children.  Children
// holding at most leafMax triangles become leaf slots; their triangles are
// copied next to each other in slot order.  Per-level prefix sums give every
// node its children's and triangles' positions, so the layout is
// deterministic.
constexpr int kNoChild = INT_MIN;

__device__ __forceinline__ int subtreeCount(const int2* range, int c)
{
    return c >= 0 ? range[c].y - range[c].x + 1 : 1;
}

__global__ void kWideCollect(const int2* __restrict__ items, int m, const int2* __restrict__ children,
                             const int2* __restrict__ range, const float* __restrict__ innerBox, int leafMax,
                             int* outCodes, int* cntI, int* cntT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) { cntI[m] = 0; cntT[m] = 0; return; }
    const int code = items[i].x;
    int C[8];
    int k;
    if (code >= 0) { const int2 c = children[code]; C[0] = c.x; C[1] = c.y; k = 2; }
    else { C[0] = code; k = 1; }
    while (k < 8) {
        int best = -1;
        float bestA = -1.0f;
        for (int phase = 0; phase < 2 && best < 0; ++phase) {
            for (int j = 0; j < k; ++j) {
                const int c = C[j];
                if (c < 0) continue;
                const int cnt = subtreeCount(range, c);
                if (phase == 0 ? cnt <= leafMax : cnt < 2) continue;
                const float A = halfArea(innerBox + 6 * static_cast<size_t>(c));
                if (A > bestA) { bestA = A; best = j; }
            }
        }
        if (best < 0) break;
        const int2 cc = children[C[best]];
        C[best] = cc.x;
        C[k++] = cc.y;
    }
    int I = 0, T = 0;
    for (int j = 0; j < 8; ++j) {
        if (j < k) {
            const int cnt = subtreeCount(range, C[j]);
            if (C[j] >= 0 && cnt > leafMax) ++I; else T += cnt;
        }
        outCodes[8 * static_cast<size_t>(i) + j] = j < k ? C[j] : kNoChild;
    }
    cntI[i] = I;
    cntT[i] = T;
}

// ---- surface-area-optimal choice of each wide node's children (the dynamic
// program of Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal on
// GPUs Through Compressed Wide BVHs", HPG 2017, with leaf slots decided by
// triangle count as above).  For a binary subtree x and j = 1..8,
// C(x, j) = the least cost of x as at most j slots of its parent:
//   C(x, 1) = A(x) cTri count(x)            when count(x) <= leafMax (a leaf slot)
//           = A(x) cNode + min_j D(x, j)     otherwise (an 8-wide node of its own)
//   D(x, j) = min_k C(left, k) + C(right, j - k)   (x's slots split between its children)
//   C(x, j) = min(C(x, j - 1), D(x, j)) for j >= 2.
// A bottom-up pass (arrival counters, as the refit) stores C and the choices;
// a wide node rooted at x then takes the slots of its best split, following
// the stored choices down.  Ties keep the fewer slots / the smaller k, so the
// tree does not depend on scheduling.
constexpr float kSahNode = 1.0f;
constexpr float kSahTri = 1.0f;   // cost of one triangle test in node visits (measured: 0.8-1.5 best of 0.1-1.5)

struct WideChoice {
    float c[9];          // C(x, 1..8) in c[1..8]
    uint8_t split[9];    // per j: 0 = fewer slots (j - 1), else k slots go to the left child
    uint8_t expandJ, expandK;   // the best split of x's own 8-wide node
};

__global__ void kWideCost(const int2* __restrict__ children, const int* __restrict__ parentInner,
                          const int* __restrict__ parentLeaf, const int2* __restrict__ range,
                          const float* __restrict__ innerBox, const float* __restrict__ leafBox, int n, int leafMax,
                          float cTri, int* arrivals, WideChoice* ch)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || n < 2) return;
    int node = parentLeaf[k];
    while (node >= 0) {
        if (atomicAdd(&arrivals[node], 1) == 0) return;   // the sibling's subtree is not done yet
        __threadfence();
        const int2 c = children[node];
        float cl[9], cr[9];
        for (int side = 0; side < 2; ++side) {
            const int x = side ? c.y : c.x;
            float* out = side ? cr : cl;
            if (x >= 0) {
                for (int j = 1; j <= 8; ++j) out[j] = __ldcg(&ch[x].c[j]);
            } else {
                const float a = halfArea(leafBox + 6 * static_cast<size_t>(~x)) * cTri;
                for (int j = 1; j <= 8; ++j) out[j] = a;
            }
        }
        WideChoice w;
        float dist[9];
        uint8_t distK[9];
        float bestD = 0.0f;
        int bestJ = 2;
        for (int j = 2; j <= 8; ++j) {
            float best = cl[1] + cr[j - 1];
            int bk = 1;
            for (int kk = 2; kk < j; ++kk) {
                const float v = cl[kk] + cr[j - kk];
                if (v < best) { best = v; bk = kk; }
            }
            dist[j] = best;
            distK[j] = static_cast<uint8_t>(bk);
            if (j == 2 || best < bestD) { bestD = best; bestJ = j; }
        }
        const int cnt = range[node].y - range[node].x + 1;
        const float A = halfArea(innerBox + 6 * static_cast<size_t>(node));
        w.c[0] = 0.0f;
        w.c[1] = cnt <= leafMax ? A * cTri * static_cast<float>(cnt) : A * kSahNode + bestD;
        w.split[0] = w.split[1] = 0;
        for (int j = 2; j <= 8; ++j) {
            if (dist[j] < w.c[j - 1]) { w.c[j] = dist[j]; w.split[j] = distK[j]; }
            else { w.c[j] = w.c[j - 1]; w.split[j] = 0; }
        }
        w.expandJ = static_cast<uint8_t>(bestJ);
        w.expandK = distK[bestJ];
        ch[node] = w;
        __threadfence();
        node = parentInner[node];
    }
}

__global__ void kWideCollectSah(const int2* __restrict__ items, int m, const int2* __restrict__ children,
                                const int2* __restrict__ range, const WideChoice* __restrict__ ch, int leafMax,
                                int* outCodes, int* cntI, int* cntT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) { cntI[m] = 0; cntT[m] = 0; return; }
    const int code = items[i].x;
    int C[8];
    int k = 0;
    if (code < 0) {
        C[k++] = code;
    } else {
        int sx[16], sj[16], sp = 0;   // pending (subtree, slots); at most 8 slots, so at most 8 pending
        const WideChoice& r = ch[code];
        const int2 c = children[code];
        sx[sp] = c.y; sj[sp++] = r.expandJ - r.expandK;
        sx[sp] = c.x; sj[sp++] = r.expandK;
        while (sp > 0 && k < 8) {
            const int x = sx[--sp];
            int j = sj[sp];
            if (x >= 0) while (j > 1 && ch[x].split[j] == 0) --j;
            if (x < 0 || j <= 1 || sp + 2 > 16) { C[k++] = x; continue; }
            const int kk = ch[x].split[j];
            const int2 cc = children[x];
            sx[sp] = cc.y; sj[sp++] = j - kk;
            sx[sp] = cc.x; sj[sp++] = kk;
        }
    }
    int I = 0, T = 0;
    for (int j = 0; j < 8; ++j) {
        if (j < k) {
            const int cnt = subtreeCount(range, C[j]);
            if (C[j] >= 0 && cnt > leafMax) ++I; else T += cnt;
        }
        outCodes[8 * static_cast<size_t>(i) + j] = j < k ? C[j] : kNoChild;
    }
    cntI[i] = I;
    cntT[i] = T;
}

__device__ __forceinline__ uint32_t wideScaleBits(uint32_t e) { return e << 23; }
// p + q * 2^(e-127) in double (exact for the magnitudes a scene has), the
// plane the traversal's fused slab test measures against
__device__ __forceinline__ double wideDecodeExact(uint32_t q, uint32_t e, float p)
{
    const double scale = __longlong_as_double(static_cast<long long>(static_cast<int>(e) - 127 + 1023) << 52);
    return static_cast<double>(p) + static_cast<double>(q) * scale;
}

// smallest biased exponent e in [1, 254] with p + 255 * 2^(e-127) >= hi
__device__ uint32_t wideExponent(float lo, float hi)
{
    const float ext = hi - lo;
    int e = 1;
    if (ext > 0.0f) e = max(1, static_cast<int>((__float_as_uint(ext) >> 23) & 0xffu) - 8);
    while (e < 254 && wideDecodeExact(255u, static_cast<uint32_t>(e), lo) < static_cast<double>(hi)) ++e;
    return static_cast<uint32_t>(e);
}

__device__ uint32_t quantLo(float v, float p, uint32_t e)
{
    const float sc = __uint_as_float(wideScaleBits(e));
    float f = floorf((v - p) / sc);
    int q = static_cast<int>(fminf(fmaxf(f, 0.0f), 255.0f));
    const double dv = static_cast<double>(v);
    while (q > 0 && wideDecodeExact(static_cast<uint32_t>(q), e, p) > dv) --q;
    while (q < 255 && wideDecodeExact(static_cast<uint32_t>(q + 1), e, p) <= dv) ++q;
    return static_cast<uint32_t>(q);
}

__device__ uint32_t quantHi(float v, float p, uint32_t e)
{
    const float sc = __uint_as_float(wideScaleBits(e));
    float f = ceilf((v - p) / sc);
    int q = static_cast<int>(fminf(fmaxf(f, 0.0f), 255.0f));
    const double dv = static_cast<double>(v);
    while (q < 255 && wideDecodeExact(static_cast<uint32_t>(q), e, p) < dv) ++q;
    while (q > 0 && wideDecodeExact(static_cast<uint32_t>(q - 1), e, p) >= dv) --q;
    return static_cast<uint32_t>(q);
}

__global__ void kWideEmit(const int2* __restrict__ items, int m, const int* __restrict__ codes,
                          const int* __restrict__ scanI, const int* __restrict__ scanT, const int2* __restrict__ range,
                          const float* __restrict__ innerBox, const float* __restrict__ leafBox,
                          const float4* __restrict__ sortedTris, int leafMax, int nextBase, int triCursor,
                          WideNode* nodes, int2* nextItems, float4* wideTris, unsigned int* errorFlag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int w = items[i].y;
    int C[8];
    int k = 0;
    float bx[8][6];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int j = 0; j < 8; ++j) {
        const int c = codes[8 * static_cast<size_t>(i) + j];
        if (c == kNoChild) break;
        C[k] = c;
        const float* b = c >= 0 ? innerBox + 6 * static_cast<size_t>(c) : leafBox + 6 * static_cast<size_t>(~c);
        for (int q = 0; q < 6; ++q) bx[k][q] = b[q];
        for (int a = 0; a < 3; ++a) { lo[a] = fminf(lo[a], b[a]); hi[a] = fmaxf(hi[a], b[3 + a]); }
        ++k;
    }
    // slot assignment: child j to slot s maximising the offset of its centre
    // towards corner s of the parent box (bit a of s set = high side of axis a)
    float pc[3];
    for (int a = 0; a < 3; ++a) pc[a] = 0.5f * (lo[a] + hi[a]);
    int slotOf[8];
    int childAt[8];
    for (int j = 0; j < 8; ++j) { slotOf[j] = -1; childAt[j] = -1; }
    for (int it = 0; it < k; ++it) {
        float bestV = -FLT_MAX;
        int bj = -1, bs = -1;
        for (int j = 0; j < k; ++j) {
            if (slotOf[j] >= 0) continue;
            float d[3];
            for (int a = 0; a < 3; ++a) d[a] = 0.5f * (bx[j][a] + bx[j][3 + a]) - pc[a];
            for (int sl = 0; sl < 8; ++sl) {
                if (childAt[sl] >= 0) continue;
                const float v = ((sl & 1) ? d[0] : -d[0]) + ((sl & 2) ? d[1] : -d[1]) + ((sl & 4) ? d[2] : -d[2]);
                if (bj < 0 || v > bestV) { bestV = v; bj = j; bs = sl; }
            }
        }
        slotOf[bj] = bs;
        childAt[bs] = bj;
    }
    uint32_t e[3];
    for (int a = 0; a < 3; ++a) e[a] = wideExponent(lo[a], hi[a]);
    WideNode nd;
    nd.px = lo[0]; nd.py = lo[1]; nd.pz = lo[2];
    nd.childBase = nextBase + scanI[i];
    nd.triBase = triCursor + scanT[i];
    uint32_t imask = 0;
    uint32_t meta[2] = {0u, 0u};
    // empty slots keep lo = 255, hi = 0 on every axis: a box inverted by the parent's whole extent, which the
    // traversal's near/far-plane test rejects without a separate validity check
    uint32_t q[6][2] = {{~0u, ~0u}, {~0u, ~0u}, {~0u, ~0u}, {0u, 0u}, {0u, 0u}, {0u, 0u}};
    int r = 0, toff = 0;
    for (int sl = 0; sl < 8; ++sl) {
        const int j = childAt[sl];
        if (j < 0) continue;
        const int c = C[j];
        const int word = sl >> 2, sh = 8 * (sl & 3);
        for (int a = 0; a < 3; ++a) {
            q[a][word] = (q[a][word] & ~(0xffu << sh)) | (quantLo(bx[j][a], lo[a], e[a]) << sh);
            q[3 + a][word] |= quantHi(bx[j][3 + a], lo[a], e[a]) << sh;
        }
        const int cnt = subtreeCount(range, c);
        if (c >= 0 && cnt > leafMax) {
            imask |= 1u << sl;
            nextItems[scanI[i] + r] = make_int2(c, nextBase + scanI[i] + r);
            ++r;
        } else {
            if (cnt > 7 || toff + cnt > 32) { atomicOr(errorFlag, 1u); continue; }
            meta[word] |= static_cast<uint32_t>(toff | (cnt << 5)) << sh;
            const int start = c >= 0 ? range[c].x : ~c;
            const size_t dst = 3 * (static_cast<size_t>(nd.triBase) + static_cast<size_t>(toff));
            for (int t = 0; t < cnt; ++t) {
                const size_t src = 3 * static_cast<size_t>(start + t);
                wideTris[dst + 3 * t] = sortedTris[src];
                wideTris[dst + 3 * t + 1] = sortedTris[src + 1];
                wideTris[dst + 3 * t + 2] = sortedTris[src + 2];
            }
            toff += cnt;
        }
    }
    nd.expImask = e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24);
    nd.meta[0] = meta[0]; nd.meta[1] = meta[1];
    nd.qlox[0] = q[0][0]; nd.qlox[1] = q[0][1];
    nd.qloy[0] = q[1][0]; nd.qloy[1] = q[1][1];
    nd.qloz[0] = q[2][0]; nd.qloz[1] = q[2][1];
    nd.qhix[0] = q[3][0]; nd.qhix[1] = q[3][1];
    nd.qhiy[0] = q[4][0]; nd.qhiy[1] = q[4][1];
    nd.qhiz[0] = q[5][0]; nd.qhiz[1] = q[5][1];
    nodes[w] = nd;
}

}  // namespace

#define BVH_CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { err = std::string("LBVH build: ") + cudaGetErrorString(e_); goto fail; } } while (0)

// Collapse the binary tree into the 8-wide tree, level by level.
static int buildWide(int n, int leafMax, const int2* children, const int2* range, const float* innerBox,
                     const float* leafBox, const float4* sortedTris, const WideChoice* choice, BvhBuildResult& out,
                     cudaStream_t st, std::string& err)
{
    int2 *itemsA = nullptr, *itemsB = nullptr;
    int *codes = nullptr, *cntI = nullptr, *cntT = nullptr;
    unsigned int* flag = nullptr;
    WideNode* scratch = nullptr;
    int rc = -1;
    int wideCount = 1, triCursor = 0, m = 1, levels = 0;
    const size_t cap = static_cast<size_t>(n > 1 ? n : 1);
    {
        BVH_CK(cudaMalloc(&itemsA, sizeof(int2) * cap));
        BVH_CK(cudaMalloc(&itemsB, sizeof(int2) * cap));
        BVH_CK(cudaMalloc(&codes, sizeof(int) * 8 * cap));
        BVH_CK(cudaMalloc(&cntI, sizeof(int) * (cap + 1)));
        BVH_CK(cudaMalloc(&cntT, sizeof(int) * (cap + 1)));
        BVH_CK(cudaMalloc(&flag, sizeof(unsigned int)));
        BVH_CK(cudaMalloc(&scratch, sizeof(WideNode) * cap));
        BVH_CK(cudaMalloc(&out.leafTris, sizeof(float4) * 3 * static_cast<size_t>(n)));
        BVH_CK(cudaMemsetAsync(flag, 0, sizeof(unsigned int), st));
        const int2 root = make_int2(n > 1 ? 0 : ~0, 0);
        BVH_CK(cudaMemcpyAsync(itemsA, &root, sizeof(int2), cudaMemcpyHostToDevice, st));
        while (m > 0) {
            const int B = 128;
            if (choice)
                kWideCollectSah<<<(m + 1 + B - 1) / B, B, 0, st>>>(itemsA, m, children, range, choice, leafMax, codes,
                                                                 cntI, cntT);
            else
                kWideCollect<<<(m + 1 + B - 1) / B, B, 0, st>>>(itemsA, m, children, range, innerBox, leafMax, codes,
                                                              cntI, cntT);
            kScanSingle<<<1, 1024, 0, st>>>(cntI, m + 1);
            kScanSingle<<<1, 1024, 0, st>>>(cntT, m + 1);
            kWideEmit<<<(m + B - 1) / B, B, 0, st>>>(itemsA, m, codes, cntI, cntT, range, innerBox, leafBox, sortedTris,
                                                     leafMax, wideCount, triCursor, scratch, itemsB, out.leafTris, flag);
            BVH_CK(cudaGetLastError());
            int tot[2] = {0, 0};
            BVH_CK(cudaMemcpyAsync(&tot[0], cntI + m, sizeof(int), cudaMemcpyDeviceToHost, st));
            BVH_CK(cudaMemcpyAsync(&tot[1], cntT + m, sizeof(int), cudaMemcpyDeviceToHost, st));
            BVH_CK(cudaStreamSynchronize(st));
            ++levels;
            wideCount += tot[0];
            triCursor += tot[1];
            m = tot[0];
            int2* t = itemsA; itemsA = itemsB; itemsB = t;
            if (static_cast<size_t>(wideCount) > cap) { err = "LBVH build: 8-wide node count exceeds its bound"; goto fail; }
        }
        unsigned int hflag = 0;
        BVH_CK(cudaMemcpyAsync(&hflag, flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        BVH_CK(cudaStreamSynchronize(st));
        if (hflag || triCursor != n) { err = "LBVH build: 8-wide collapse lost triangles"; goto fail; }
        BVH_CK(cudaMalloc(&out.wnodes, sizeof(WideNode) * wideCount));
        BVH_CK(cudaMemcpyAsync(out.wnodes, scratch, sizeof(WideNode) * wideCount, cudaMemcpyDeviceToDevice, st));
        BVH_CK(cudaStreamSynchronize(st));
        out.nodeCount = wideCount;
        out.depth = levels;
        rc = 0;
    }
fail:
    cudaFree(itemsA); cudaFree(itemsB); cudaFree(codes); cudaFree(cntI); cudaFree(cntT); cudaFree(flag);
    cudaFree(scratch);
    if (rc != 0) {
        cudaFree(out.leafTris); out.leafTris = nullptr;
        cudaFree(out.wnodes); out.wnodes = nullptr;
    }
    return rc;
}

// PLOC hierarchy over the Morton-sorted triangles `sortedMorton`: fills
// children / parentInner / parentLeaf / range like kKarras, with the leaves in
// depth-first order, and that order's triangles in `sortedDfs`.  *depth = the
// deepest leaf's depth (root = 1).
static int buildPloc(const TriangleData* dTris, const int* sortedMorton, int n, int radius, int2* children,
                     int* parentInner, int* parentLeaf, int2* range, int* sortedDfs, int* depth, cudaStream_t st,
                     std::string& err)
{
    Cluster *cA = nullptr, *cB = nullptr;
    int *nn = nullptr, *counts = nullptr, *firstInner = nullptr, *parentMorton = nullptr, *dDepth = nullptr;
    int2* tileSums = nullptr;
    int rc = -1;
    const int inner = n - 1;
    const int maxTiles = (n + kPlocTile - 1) / kPlocTile;
    {
        BVH_CK(cudaMalloc(&cA, sizeof(Cluster) * n));
        BVH_CK(cudaMalloc(&cB, sizeof(Cluster) * n));
        BVH_CK(cudaMalloc(&nn, sizeof(int) * n));
        BVH_CK(cudaMalloc(&counts, sizeof(int) * inner));
        BVH_CK(cudaMalloc(&firstInner, sizeof(int) * inner));
        BVH_CK(cudaMalloc(&parentMorton, sizeof(int) * n));
        BVH_CK(cudaMalloc(&dDepth, sizeof(int)));
        BVH_CK(cudaMalloc(&tileSums, sizeof(int2) * (maxTiles + 1)));
        const int B = 256;
        kPlocInit<<<(n + B - 1) / B, B, 0, st>>>(dTris, sortedMorton, n, cA);
        int m = n, nextId = n - 2, rounds = 0;
        while (m > 1) {
            const int tiles = (m + kPlocTile - 1) / kPlocTile;
            kPlocNearest<<<(m + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, st>>>(cA, m, radius, nn);
            kPlocCount<<<tiles, kPlocBlock, 0, st>>>(nn, m, tileSums);
            kPlocScanTiles<<<1, 1024, 0, st>>>(tileSums, tiles);
            kPlocCompact<<<tiles, kPlocBlock, 0, st>>>(cA, nn, m, tileSums, nextId, cB, children, counts);
            BVH_CK(cudaGetLastError());
            int2 tot = make_int2(0, 0);
            BVH_CK(cudaMemcpyAsync(&tot, tileSums + tiles, sizeof(int2), cudaMemcpyDeviceToHost, st));
            BVH_CK(cudaStreamSynchronize(st));
            if (tot.y <= 0 || tot.x != m - tot.y || tot.y > nextId + 1 || ++rounds > n) {
                err = "PLOC build: a clustering round merged no pair";
                goto fail;
            }
            m = tot.x;
            nextId -= tot.y;
            Cluster* t = cA; cA = cB; cB = t;
        }
        if (nextId != -1) { err = "PLOC build: merge count differs from n-1"; goto fail; }
        BVH_CK(cudaMemsetAsync(dDepth, 0, sizeof(int), st));
        kPlocParents<<<(inner + B - 1) / B, B, 0, st>>>(children, inner, parentInner, parentMorton);
        kPlocFirstInner<<<(inner + B - 1) / B, B, 0, st>>>(children, parentInner, counts, inner, firstInner, dDepth);
        kPlocRelabel<<<(n + B - 1) / B, B, 0, st>>>(children, counts, firstInner, parentMorton, sortedMorton, n, range,
                                                    sortedDfs, parentLeaf);
        kPlocLeafCodes<<<(inner + B - 1) / B, B, 0, st>>>(children, counts, firstInner, inner);
        BVH_CK(cudaGetLastError());
        BVH_CK(cudaMemcpyAsync(depth, dDepth, sizeof(int), cudaMemcpyDeviceToHost, st));
        BVH_CK(cudaStreamSynchronize(st));
        rc = 0;
    }
fail:
    cudaFree(cA); cudaFree(cB); cudaFree(nn); cudaFree(counts); cudaFree(firstInner); cudaFree(parentMorton);
    cudaFree(dDepth); cudaFree(tileSums);
    return rc;
}

// Steps 1-3: per-triangle centroids and their bounds, 63-bit Morton codes (keysA / valsA = triangle index), and
// the stable LSD radix sort of (code, index) over 16 passes of 4-bit digits.  *sortedKeys / *sortedVals name the
// ping-pong buffers holding the sorted pairs, *spareKeys / *spareVals the other two.  bounds holds 6 words and
// hist kDigits * ceil(n / kSortTile) ints.
int launchMortonSort(const TriangleData* dTris, int n, float4* cen, unsigned int* bounds, unsigned long long* keysA,
                     unsigned long long* keysB, int* valsA, int* valsB, int* hist, cudaStream_t st,
                     unsigned long long** sortedKeys, unsigned long long** spareKeys, int** sortedVals,
                     int** spareVals, std::string& err)
{
    const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    cudaError_t e = cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { err = std::string("LBVH build: ") + cudaGetErrorString(e); return -1; }
    const int B = 256, G = (n + B - 1) / B;
    const int numTiles = (n + kSortTile - 1) / kSortTile;
    kTriPrep<<<G, B, 0, st>>>(dTris, n, cen, bounds);
    kMorton<<<G, B, 0, st>>>(cen, n, bounds, keysA, valsA);
    unsigned long long *kin = keysA, *kout = keysB;
    int *vin = valsA, *vout = valsB;
    for (int shift = 0; shift < 64; shift += 4) {
        kRadixHist<<<numTiles, kSortThreads, 0, st>>>(kin, n, shift, numTiles, hist);
        kScanSingle<<<1, 1024, 0, st>>>(hist, kDigits * numTiles);
        kRadixScatter<<<numTiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, numTiles, hist);
        unsigned long long* tk = kin; kin = kout; kout = tk;
        int* tv = vin; vin = vout; vout = tv;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) { err = std::string("LBVH build: ") + cudaGetErrorString(e); return -1; }
    *sortedKeys = kin; *spareKeys = kout; *sortedVals = vin; *spareVals = vout;
    return 0;
}

// The Morton codes and sorted order the build produces for host triangles (a check of the integer steps).
int lbvhMortonOrder(const TriangleData* hostTris, int n, unsigned long long* hostKeys, int* hostSorted,
                    std::string& err)
{
    if (n <= 0 || !hostTris) { err = "bte_debug_lbvh_order: no triangles"; return -1; }
    TriangleData* tris = nullptr;
    float4* cen = nullptr;
    unsigned int* bounds = nullptr;
    unsigned long long *keysA = nullptr, *keysB = nullptr, *kin = nullptr, *kout = nullptr;
    int *valsA = nullptr, *valsB = nullptr, *hist = nullptr, *vin = nullptr, *vout = nullptr;
    const int numTiles = (n + kSortTile - 1) / kSortTile;
    int rc = -1;
    cudaStream_t st = nullptr;
    auto okc = [&](cudaError_t e) {
        if (e != cudaSuccess) err = std::string("bte_debug_lbvh_order: ") + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    if (okc(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) &&
        okc(cudaMalloc(&tris, sizeof(TriangleData) * n)) && okc(cudaMalloc(&cen, sizeof(float4) * n)) &&
        okc(cudaMalloc(&bounds, sizeof(unsigned int) * 6)) && okc(cudaMalloc(&keysA, sizeof(unsigned long long) * n)) &&
        okc(cudaMalloc(&keysB, sizeof(unsigned long long) * n)) && okc(cudaMalloc(&valsA, sizeof(int) * n)) &&
        okc(cudaMalloc(&valsB, sizeof(int) * n)) && okc(cudaMalloc(&hist, sizeof(int) * kDigits * numTiles)) &&
        okc(cudaMemcpyAsync(tris, hostTris, sizeof(TriangleData) * n, cudaMemcpyHostToDevice, st))) {
        // the codes before sorting are kMorton's output: copy them out of keysA before the first pass moves them
        const int B = 256, G = (n + B - 1) / B;
        const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        if (okc(cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st))) {
            kTriPrep<<<G, B, 0, st>>>(tris, n, cen, bounds);
            kMorton<<<G, B, 0, st>>>(cen, n, bounds, keysA, valsA);
            if (okc(cudaGetLastError()) &&
                okc(cudaMemcpyAsync(hostKeys, keysA, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, st)) &&
                okc(cudaStreamSynchronize(st)) &&
                launchMortonSort(tris, n, cen, bounds, keysA, keysB, valsA, valsB, hist, st, &kin, &kout, &vin, &vout,
                                 err) == 0 &&
                okc(cudaMemcpyAsync(hostSorted, vin, sizeof(int) * n, cudaMemcpyDeviceToHost, st)) &&
                okc(cudaStreamSynchronize(st)))
                rc = 0;
        }
    }
    cudaFree(tris); cudaFree(cen); cudaFree(bounds); cudaFree(keysA); cudaFree(keysB); cudaFree(valsA); cudaFree(valsB);
    cudaFree(hist);
    if (st) cudaStreamDestroy(st);
    return rc;
}

int buildLbvh(const TriangleData* dTris, int n, int maxLeaf, int width, int builder, int radius, int wideCollapse,
              BvhBuildResult& out, cudaStream_t st, std::string& err)
{
    WideChoice* choice = nullptr;
    out = BvhBuildResult{};
    if (n <= 0) return 0;
    if (width != 2 && width != 8) { err = "LBVH build: tree width must be 2 or 8"; return -1; }
    if (n > kLeafStartMask) { err = "LBVH build: too many triangles for the leaf encoding"; return -1; }
    if (maxLeaf < 1) maxLeaf = 1;
    if (maxLeaf > kMaxLeafTris) maxLeaf = kMaxLeafTris;
    float4* cen = nullptr;
    unsigned int* bounds = nullptr;
    unsigned long long *keysA = nullptr, *keysB = nullptr;
    int *valsA = nullptr, *valsB = nullptr, *hist = nullptr;
    int2* children = nullptr;
    int *parentInner = nullptr, *parentLeaf = nullptr, *arrivals = nullptr, *collapsed = nullptr;
    float *innerBox = nullptr, *leafBox = nullptr, *cost = nullptr;
    int2* range = nullptr;
    float4* sorted = nullptr;   // triangles in sorted (binary leaf) order
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int numTiles = (n + kSortTile - 1) / kSortTile;
    const int inner = n > 1 ? n - 1 : 1;
    {
        BVH_CK(cudaEventCreate(&e0));
        BVH_CK(cudaEventCreate(&e1));
        BVH_CK(cudaEventRecord(e0, st));
        BVH_CK(cudaMalloc(&cen, sizeof(float4) * n));
        BVH_CK(cudaMalloc(&bounds, sizeof(unsigned int) * 6));
        BVH_CK(cudaMalloc(&keysA, sizeof(unsigned long long) * n));
        BVH_CK(cudaMalloc(&keysB, sizeof(unsigned long long) * n));
        BVH_CK(cudaMalloc(&valsA, sizeof(int) * n));
        BVH_CK(cudaMalloc(&valsB, sizeof(int) * n));
        BVH_CK(cudaMalloc(&hist, sizeof(int) * kDigits * numTiles));
        BVH_CK(cudaMalloc(&children, sizeof(int2) * inner));
        BVH_CK(cudaMalloc(&parentInner, sizeof(int) * inner));
        BVH_CK(cudaMalloc(&parentLeaf, sizeof(int) * n));
        BVH_CK(cudaMalloc(&arrivals, sizeof(int) * inner));
        BVH_CK(cudaMalloc(&collapsed, sizeof(int) * inner));
        BVH_CK(cudaMalloc(&cost, sizeof(float) * inner));
        BVH_CK(cudaMalloc(&range, sizeof(int2) * inner));
        BVH_CK(cudaMalloc(&innerBox, sizeof(float) * 6 * inner));
        BVH_CK(cudaMalloc(&leafBox, sizeof(float) * 6 * n));
        BVH_CK(cudaMalloc(&sorted, sizeof(float4) * 3 * static_cast<size_t>(n)));
        if (width == 2) BVH_CK(cudaMalloc(&out.nodes, sizeof(BvhNode) * inner));
        BVH_CK(cudaMemsetAsync(arrivals, 0, sizeof(int) * inner, st));
        const int B = 256, G = (n + B - 1) / B;
        unsigned long long *kin = nullptr, *kout = nullptr;
        int *vin = nullptr, *vout = nullptr;
        if (launchMortonSort(dTris, n, cen, bounds, keysA, keysB, valsA, valsB, hist, st, &kin, &kout, &vin, &vout,
                             err) != 0)
            goto fail;
        out.builder = 0;
        if (n > 1 && builder == 1) {
            int depth = 0;
            if (buildPloc(dTris, vin, n, radius, children, parentInner, parentLeaf, range, vout, &depth, st, err) != 0)
                goto fail;
            if (width == 8 || depth - 1 <= kTraversalStack) {   // else the binary walk's stack could overflow
                int* tv = vin; vin = vout; vout = tv;
                out.builder = 1;
            }
        }
        if (n > 1 && out.builder == 0) {
            kKarras<<<(n - 1 + B - 1) / B, B, 0, st>>>(kin, n, children, parentInner, parentLeaf, range);
        }
        kRefit<<<G, B, 0, st>>>(dTris, vin, n, children, parentInner, parentLeaf, range, sorted, innerBox, leafBox,
                                arrivals, cost, collapsed, maxLeaf);
        BVH_CK(cudaGetLastError());
        out.width = width;
        if (width == 8) {
            const int wideLeaf = maxLeaf < kWideLeafMax ? maxLeaf : kWideLeafMax;
            if (wideCollapse == 1 && n > 1) {   // surface-area-optimal children of each wide node
                BVH_CK(cudaMalloc(&choice, sizeof(WideChoice) * inner));
                BVH_CK(cudaMemsetAsync(arrivals, 0, sizeof(int) * inner, st));
                kWideCost<<<G, B, 0, st>>>(children, parentInner, parentLeaf, range, innerBox, leafBox, n, wideLeaf,
                                           kSahTri, arrivals, choice);
                BVH_CK(cudaGetLastError());
            }
            if (buildWide(n, wideLeaf, children, range, innerBox, leafBox, sorted, choice, out, st, err) != 0)
                goto fail;
            BVH_CK(cudaEventRecord(e1, st));
            BVH_CK(cudaEventSynchronize(e1));
            BVH_CK(cudaEventElapsedTime(&out.msBuild, e0, e1));
            cudaFree(sorted);
            sorted = nullptr;
        } else {
            if (n > 1) kEmitNodes<<<(n - 1 + B - 1) / B, B, 0, st>>>(children, innerBox, leafBox, range, collapsed, n, out.nodes);
            BVH_CK(cudaGetLastError());
            BVH_CK(cudaEventRecord(e1, st));
            BVH_CK(cudaEventSynchronize(e1));
            BVH_CK(cudaEventElapsedTime(&out.msBuild, e0, e1));
            out.leafTris = sorted;
            sorted = nullptr;
            out.nodeCount = n > 1 ? n - 1 : 0;
        }
        out.rootIsLeaf = n == 1 ? 1 : 0;
        out.rootCode = ~0;
        if (width == 2 && n > 1) {   // a scene small enough to be one leaf
            int rootCollapsed = 0;
            BVH_CK(cudaMemcpyAsync(&rootCollapsed, collapsed, sizeof(int), cudaMemcpyDeviceToHost, st));
            BVH_CK(cudaStreamSynchronize(st));
            if (rootCollapsed) { out.rootIsLeaf = 1; out.rootCode = ~((n - 1) << kLeafCountShift); }
        }
    }
    cudaFree(cen); cudaFree(bounds); cudaFree(keysA); cudaFree(keysB); cudaFree(valsA); cudaFree(valsB); cudaFree(hist);
    cudaFree(children); cudaFree(parentInner); cudaFree(parentLeaf); cudaFree(arrivals); cudaFree(innerBox);
    cudaFree(leafBox); cudaFree(collapsed); cudaFree(cost); cudaFree(range); cudaFree(choice);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    return 0;
fail:
    cudaFree(cen); cudaFree(bounds); cudaFree(keysA); cudaFree(keysB); cudaFree(valsA); cudaFree(valsB); cudaFree(hist);
    cudaFree(children); cudaFree(parentInner); cudaFree(parentLeaf); cudaFree(arrivals); cudaFree(innerBox);
    cudaFree(leafBox); cudaFree(collapsed); cudaFree(cost); cudaFree(range); cudaFree(sorted); cudaFree(choice);
    cudaFree(out.leafTris); cudaFree(out.nodes); cudaFree(out.wnodes);
    out = BvhBuildResult{};
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return -1;
}

}  // namespace bte
