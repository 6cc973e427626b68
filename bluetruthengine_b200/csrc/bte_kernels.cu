// bte_kernels.cu -- wavefront stage kernels (sm_100a).
//
//   generate -> [extend -> shade -> connect] x maxDepth -> present
//
// One frame is a fixed launch sequence with no host round trip: every stage
// reads its work count from a per-bounce device counter, so the sequence can
// be replayed as a CUDA graph.  This replaces the reference's host-driven
// loop (src/host/wavefront_host.cu:155-236), which copies counters to the
// host and synchronises several times per bounce.
//
// Path state is structure-of-arrays with 16-byte records (one 128-bit load or
// store per field) instead of the reference's 12-byte Float3 arrays
// (include/wavefront/wavefront_buffers.h:40-90).  Queue appends are
// warp-aggregated (one atomic per coalesced group).  NEE shadow rays live in
// fixed per-path slots (area, spotlights, env); connect clears the visibility
// bit of occluded slots and the next shade (or present) adds the surviving
// contributions in the reference's megakernel order, which makes the result
// deterministic where the reference races float atomicAdds
// (src/wavefront/ray_connect.cu:67-69).
#include "bte_kernels.h"
#include "bte_shade.cuh"
#include "bte_trace.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace bte {

namespace {

BTE_DI int appendCoalesced(int* counter)
{
    cg::coalesced_group g = cg::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, static_cast<int>(g.size()));
    base = g.shfl(base, 0);
    return base + static_cast<int>(g.thread_rank());
}

// warp-aggregated append into one of several counters (lanes grouped by key)
BTE_DI int appendKeyed(int* counters, int key)
{
    const unsigned active = __activemask();
    const unsigned same = __match_any_sync(active, key);
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(same) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counters + key, __popc(same));
    base = __shfl_sync(same, base, leader);
    return base + __popc(same & ((1u << lane) - 1u));
}

// bucket of a path for material-sorted shading: 0 miss, else the BSDF type of the hit triangle
BTE_DI int sortKey(const DevScene& s, int tri)
{
    const int key = tri < 0 ? 0 : s.bsdfs[s.triBsdfIds[tri]].type;
    return (key >= 0 && key < kSortKeys) ? key : 0;
}
BTE_DI void sortAppend(const DevScene& s, const DevPaths& P, int bounce, int idx, int tri)
{
    const int k = sortKey(s, tri);
    P.sortQueue[static_cast<size_t>(k) * P.count + appendKeyed(P.sortCount + bounce * kSortKeys, k)] = idx;
}
// extend's hand-over to shade: the bucket append, or -- on a path-ordered bounce -- the path's key, from which
// the ordered compaction builds the buckets
BTE_DI void bucketPath(const DevScene& s, const DevPaths& P, int bounce, int idx, int tri)
{
    if (!P.sortQueue) return;
    if (bounce < P.orderBounces) P.pathKey[idx] = static_cast<uint8_t>(sortKey(s, tri));
    else sortAppend(s, P, bounce, idx, tri);
}

BTE_DI V3 xyz(float4 a) { return v3(a.x, a.y, a.z); }

// The scene of a path: the kernel's own scene, or -- in one launch sequence over several scenes' views
// (DevPaths.scenes) -- the path's entry of the frame's scene table.
template <bool Multi>
BTE_DI const DevScene& sceneOf(const DevScene& s, const DevPaths& P, int path)
{
    if constexpr (Multi) return P.scenes[P.pathScene[path]];
    else return s;
}

// Whether bounce `bounce` walks its queue in ray-bin order (same answer in shade, kRayBins, kRayScatter, extend).
BTE_DI bool raySorted(const DevPaths& P, int bounce, int count)
{
    return P.raySortBits > 0 && bounce >= 1 && bounce <= P.raySortBounces && count >= kRaySortMinRays;
}
BTE_DI int rayBinCount(const DevPaths& P) { return 8 << (3 * P.raySortBits); }
BTE_DI uint32_t spreadBits3(uint32_t v)   // bit i of v -> bit 3i (v < 32)
{
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) x |= ((v >> i) & 1u) << (3 * i);
    return x;
}
// bin of a ray: direction octant in the high bits, then the Morton code of its origin cell
BTE_DI int rayBinOf(const DevPaths& P, float sceneMaxAbs, float4 o, float4 d)
{
    const int bits = P.raySortBits;
    const float m = sceneMaxAbs > 0.0f ? sceneMaxAbs : 1.0f;
    const float scale = static_cast<float>(1 << bits) / (2.0f * m);
    const int top = (1 << bits) - 1;
    const int cx = min(max(static_cast<int>((o.x + m) * scale), 0), top);
    const int cy = min(max(static_cast<int>((o.y + m) * scale), 0), top);
    const int cz = min(max(static_cast<int>((o.z + m) * scale), 0), top);
    const uint32_t cell = (spreadBits3(static_cast<uint32_t>(cx)) << 2) | (spreadBits3(static_cast<uint32_t>(cy)) << 1) |
                          spreadBits3(static_cast<uint32_t>(cz));
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return static_cast<int>((oct << (3 * bits)) | cell);
}

// The wavefront stops at the first bounce whose queue holds fewer than tailPaths paths; kTail then
// finishes those paths one thread each (the few long paths no longer pay a launch per bounce).
BTE_DI bool tailTakesOver(const DevPaths& P, int bounce)
{
    return P.tailPaths > 0 && P.rayCount[bounce] < P.tailPaths;
}

// Adds the contributions of the visible NEE slots in slot order and clears the mask.
BTE_DI V3 resolveShadows(const DevPaths& P, int idx, V3 L)
{
    const uint32_t mask = P.shMask[idx];
    if (mask != 0u) {
        for (int s = 0; s < P.slots; ++s) {
            if (mask & (1u << s)) {
                const float4 c = P.shContrib[static_cast<size_t>(idx) * P.slots + s];
                L = add3(L, v3(c.x, c.y, c.z));
            }
        }
        P.shMask[idx] = 0u;
    }
    return L;
}

}  // namespace

// ---------------------------------------------------------------- generate
// src/wavefront/ray_generate.cu:42-80.  Path i covers pixel i % (W*H) and
// sample frameIndex + i / (W*H).
__global__ void __launch_bounds__(256) kGenerate(DevPaths P, FrameParams f)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) P.rayCount[0] = P.count;
    if (i >= P.count) return;
    int width = f.width, height = f.height, local = i;
    uint32_t frameIndex;
    const CameraData* cam = &f.cam;
    float tanHalf = f.tanHalf;
    if (f.viewCount > 0) {   // batched views: find the view holding path i
        int v = 0;
        while (v + 1 < f.viewCount && i >= f.views[v + 1].pathOffset) ++v;
        const ViewDesc& vd = f.views[v];
        width = vd.width; height = vd.height; local = i - vd.pathOffset;
        frameIndex = vd.frameIndex;
        cam = &vd.cam;
        tanHalf = vd.tanHalf;
        if (P.pathScene) P.pathScene[i] = static_cast<uint8_t>(vd.scene);
    } else {
        frameIndex = *f.frameIndex;
    }
    const int wh = width * height;
    const int pix = local % wh;
    const int s = local / wh;
    const int px = pix % width, py = pix / width;
    uint32_t rng = rngSeed(static_cast<uint32_t>(pix), frameIndex + static_cast<uint32_t>(s));
    const float jx = rngNext(rng) - 0.5f;
    const float jy = rngNext(rng) - 0.5f;
    V3 o, d;
    primaryRay(px, py, width, height, *cam, tanHalf, jx, jy, o, d);
    P.o[i] = make_float4(o.x, o.y, o.z, __uint_as_float(rng));
    P.d[i] = make_float4(d.x, d.y, d.z, 1.0f);
    P.tp[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.L[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(1u << 16));
    P.queue[0][i] = i;
    P.shMask[i] = 0u;
}

// ---------------------------------------------------------------- extend
// src/wavefront/ray_extend.cu:49-72 with src/optix_programs.cu:110-148 moved
// to shade (the hit record is t, u, v, triangle).
template <int Width>
__global__ void __launch_bounds__(256) kExtend(DevScene s, DevPaths P, int bounce)
{
    const int count = P.rayCount[bounce];
    if (tailTakesOver(P, bounce)) return;
    const int* __restrict__ q = raySorted(P, bounce, count) ? P.sortedQueue : P.queue[bounce & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < count; slot += stride) {
        const int idx = q[slot];
        const float4 o = P.o[idx];
        const float4 d = P.d[idx];
        const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, s.sceneMaxAbs);
        float t = 0.0f, u = 0.0f, v = 0.0f;
        const int tri = traceClosestW<Width>(s, r, kEps, 1e30f, t, u, v, P.errorFlags);
        P.hit[idx] = make_float4(t, u, v, __int_as_float(tri));
        if (P.hitLog) P.hitLog[static_cast<size_t>(idx) * P.maxDepth + bounce] = tri;
        bucketPath(s, P, bounce, idx, tri);
    }
}

// ---------------------------------------------------------------- shade
// src/wavefront/ray_shade.cu:103-183 (rt_optix_shading.cuh:412-447 order).
// One path's shading at `bounce` (src/wavefront/ray_shade.cu:103-183, rt_optix_shading.cuh:412-447
// order): pending shadow contributions, emitter/env hit, NEE records in the path's slots, scatter,
// roulette; writes the path state back.  Shadow records are queued for kConnect when queueShadows,
// else left in the slots (shMask) for the caller to trace.  Returns whether the path continues.
BTE_DI bool shadePath(const DevScene& s, const DevPaths& P, const FrameParams& f, int bounce, int idx, bool queueShadows)
{
    const float4 o4 = P.o[idx], d4 = P.d[idx], tp4 = P.tp[idx], L4 = P.L[idx];
    uint32_t rng = __float_as_uint(o4.w);
    PathReg p;
    p.o = xyz(o4); p.d = xyz(d4); p.tp = xyz(tp4); p.L = xyz(L4);
    p.eta = d4.w;
    p.brdfPdf = tp4.w;
    const uint32_t bits = __float_as_uint(L4.w);
    p.bounce = static_cast<int>(bits & 0xffffu);
    p.specular = ((bits >> 16) & 1u) != 0u;

    p.L = resolveShadows(P, idx, p.L);

    const float4 hv = P.hit[idx];
    const int tri = __float_as_int(hv.w);
    if (tri < 0) {
        if (bounce == 0 && P.aovAlbedo) {
            P.aovAlbedo[idx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            P.aovNormal[idx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        accumulateEnvHit(s, p);
        P.L[idx] = make_float4(p.L.x, p.L.y, p.L.z, L4.w);
        return false;
    }
    // closest-hit attributes, src/optix_programs.cu:121-140
    HitReg h;
    h.tri = tri;
    {
        const float t = hv.x, u = hv.y, v = hv.z;
        const float w0 = 1.0f - u - v;
        const TriangleData& T = s.tris[tri];
        h.p = v3(p.o.x + t * p.d.x, p.o.y + t * p.d.y, p.o.z + t * p.d.z);
        h.n = normalize3(v3(w0 * T.n0.x + u * T.n1.x + v * T.n2.x, w0 * T.n0.y + u * T.n1.y + v * T.n2.y,
                            w0 * T.n0.z + u * T.n1.z + v * T.n2.z));
        h.u = w0 * T.uv0.x + u * T.uv1.x + v * T.uv2.x;
        h.v = w0 * T.uv0.y + u * T.uv1.y + v * T.uv2.y;
    }
    const Bsdf b = loadBsdf(s, tri, h.u, h.v);
    bool featPending = false;
    if (P.aovAlbedo && (bounce == 0 || ((bits >> 17) & 1u) != 0u)) {
        // denoiser features: the material colour and shading normal of the first hit that is not a perfect
        // mirror or dielectric, seen through the mirrors and dielectrics in front of it (their colours multiplied
        // in: a mirror's tint, 1 for a dielectric).  While a path has met only such surfaces, the last one's
        // normal and the product so far stand, and bit 17 of the packed bounce word marks the path as pending.
        const float4 prev = bounce == 0 ? make_float4(1.0f, 1.0f, 1.0f, 0.0f) : P.aovAlbedo[idx];
        const V3 c = b.type == BSDF_Dielectric ? v3(1.0f, 1.0f, 1.0f) : v3(b.p0.x, b.p0.y, b.p0.z);
        P.aovAlbedo[idx] = make_float4(prev.x * c.x, prev.y * c.y, prev.z * c.z, 0.0f);
        P.aovNormal[idx] = make_float4(h.n.x, h.n.y, h.n.z, 0.0f);
        featPending = !bsdfIsDiffuseClass(b.type);
    }
    if (s.emitterFlags[tri] != 0) accumulateEmitterHit(s, p, h);

    const Frame fr = makeFrame(h.n);
    const V3 wiLocal = toLocal(fr, mul3(p.d, -1.0f));
    if (bsdfIsDiffuseClass(b.type)) {
        p.specular = false;
        uint32_t newMask = 0u;
        ShadowRec sr;
        const size_t base = static_cast<size_t>(idx) * P.slots;
        if (prepareArea(s, p, rng, h, b, wiLocal, fr, sr)) {
            P.shDir[base] = make_float4(sr.d.x, sr.d.y, sr.d.z, sr.tmax);
            P.shContrib[base] = make_float4(sr.c.x, sr.c.y, sr.c.z, 0.0f);
            newMask |= 1u;
            if (queueShadows) P.shadowQueue[appendCoalesced(P.shadowCount + bounce)] = static_cast<int>(base);
        }
        for (int si = 0; si < s.spotCount; ++si) {
            if (prepareSpot(s, p, h, b, si, wiLocal, fr, sr)) {
                P.shDir[base + 1 + si] = make_float4(sr.d.x, sr.d.y, sr.d.z, sr.tmax);
                P.shContrib[base + 1 + si] = make_float4(sr.c.x, sr.c.y, sr.c.z, 0.0f);
                newMask |= 1u << (1 + si);
                if (queueShadows) P.shadowQueue[appendCoalesced(P.shadowCount + bounce)] = static_cast<int>(base + 1 + si);
            }
        }
        if (prepareEnv(s, p, rng, h, b, wiLocal, fr, sr)) {
            const int es = P.slots - 1;
            P.shDir[base + es] = make_float4(sr.d.x, sr.d.y, sr.d.z, sr.tmax);
            P.shContrib[base + es] = make_float4(sr.c.x, sr.c.y, sr.c.z, 0.0f);
            newMask |= 1u << es;
            if (queueShadows) P.shadowQueue[appendCoalesced(P.shadowCount + bounce)] = static_cast<int>(base + es);
        }
        if (newMask != 0u) {
            P.shOrigin[idx] = make_float4(h.p.x, h.p.y, h.p.z, 0.0f);
            P.shMask[idx] = newMask;
        }
    } else {
        p.specular = true;
    }
    scatter(p, rng, h, b, wiLocal, fr);
    const bool alive = roulette(p, rng, f.rrStart);
    if (alive) p.bounce++;
    P.o[idx] = make_float4(p.o.x, p.o.y, p.o.z, __uint_as_float(rng));
    P.d[idx] = make_float4(p.d.x, p.d.y, p.d.z, p.eta);
    P.tp[idx] = make_float4(p.tp.x, p.tp.y, p.tp.z, p.brdfPdf);
    P.L[idx] = make_float4(p.L.x, p.L.y, p.L.z,
                           __uint_as_float(static_cast<uint32_t>(p.bounce) | (p.specular ? (1u << 16) : 0u) |
                                           (featPending ? (1u << 17) : 0u)));
    return alive;
}

// Register budget by the residency knob: 2 -> 96, 3 -> 72, 4 -> 64 registers per thread, i.e. 2, 3 or 4 resident
// blocks of 256 threads and 5, 7 or 8 of the default 128 (72 registers against 80: 1.1% faster per frame on the
// 1080p bench scene, although 72 spill a little).
template <int MinBlocks>
constexpr int shadeRegisters() { return MinBlocks == 2 ? 96 : MinBlocks == 3 ? 72 : 64; }
template <int MinBlocks, bool Multi>
__global__ void __maxnreg__(shadeRegisters<MinBlocks>()) kShade(DevScene s, DevPaths P, FrameParams f, int bounce)
{
    const int count = P.rayCount[bounce];
    if (tailTakesOver(P, bounce)) return;
    int* qn = P.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    int bucketEnd[kSortKeys];
    if (P.sortQueue) {
        int run = 0;
#pragma unroll
        for (int k = 0; k < kSortKeys; ++k) { run += P.sortCount[bounce * kSortKeys + k]; bucketEnd[k] = run; }
    }
    const int* __restrict__ q = P.queue[bounce & 1];
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < count; slot += stride) {
        int idx;
        if (P.sortQueue) {
            int k = 0, start = 0;
#pragma unroll
            for (int j = 0; j < kSortKeys - 1; ++j)
                if (slot >= bucketEnd[j]) { k = j + 1; start = bucketEnd[j]; }
            idx = P.sortQueue[static_cast<size_t>(k) * P.count + (slot - start)];
        } else {
            idx = q[slot];
        }
        const DevScene& ss = sceneOf<Multi>(s, P, idx);
        const bool alive = shadePath(ss, P, f, bounce, idx, true);
        if (bounce + 1 < P.orderBounces) {   // the ordered compaction builds the next queue
            P.pathKey[idx] = alive && bounce + 1 < P.maxDepth ? kKeyNext : kKeyDead;
        } else if (alive && bounce + 1 < P.maxDepth) {
            const int next = appendCoalesced(P.rayCount + bounce + 1);
            qn[next] = idx;
            if (P.raySortBits > 0 && bounce + 1 <= P.raySortBounces) {
                const int bin = rayBinOf(P, ss.sceneMaxAbs, P.o[idx], P.d[idx]);
                P.rayBin[next] = bin;
                appendKeyed(P.binCount + static_cast<size_t>(bounce + 1) * rayBinCount(P), bin);
            }
        }
    }
}

// Bin counts of a bounce -> bin starts (exclusive scan in place; one block, each thread a run of bins).
__global__ void __launch_bounds__(1024) kRayBins(DevPaths P, int bounce)
{
    const int count = P.rayCount[bounce];
    if (!raySorted(P, bounce, count)) return;
    const int nb = rayBinCount(P);
    int* c = P.binCount + static_cast<size_t>(bounce) * nb;
    __shared__ int part[1024];
    const int per = (nb + 1023) / 1024;
    const int lo = min(static_cast<int>(threadIdx.x) * per, nb), hi = min(lo + per, nb);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += c[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = static_cast<int>(threadIdx.x) >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0;
    for (int i = lo; i < hi; ++i) {
        const int v = c[i];
        c[i] = run;
        run += v;
    }
}

// The bounce's queue in bin order (order inside a bin is arbitrary: results do not depend on queue order).
__global__ void __launch_bounds__(256) kRayScatter(DevPaths P, int bounce)
{
    const int count = P.rayCount[bounce];
    if (!raySorted(P, bounce, count)) return;
    int* starts = P.binCount + static_cast<size_t>(bounce) * rayBinCount(P);
    const int* __restrict__ q = P.queue[bounce & 1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        P.sortedQueue[appendKeyed(starts, P.rayBin[i])] = q[i];
}

// ---------------------------------------------------------------- path-ordered queues
// One launch per bounce and selection: a stable counting sort of the paths 0 .. count-1 by pathKey into the
// material buckets after extend (keys 0 .. kSortKeys-1 into sortQueue's bucket regions, totals into sortCount)
// or the next bounce's queue after shade (key kKeyNext into queue[(bounce + 1) & 1], total into
// rayCount[bounce + 1]); inside a key the paths keep index order.  A tile is kOrderTile consecutive paths, 32 per
// thread of a 256-thread block (two 16-byte loads of their keys; pathKey is padded to whole tiles).  Tiles are
// taken in order from a ticket counter and find their output offsets by decoupled look-back (Merrill & Garland
// 2016): each publishes its per-key counts, then sums its predecessors' published words back to the first
// inclusive one.  A predecessor holds an earlier ticket, so it is running or done and its word arrives; the wait
// is bounded all the same (error flag bit 2; the offsets stay in range).  One warp per key reads 128 predecessors'
// words per round.  The tile's paths are staged in shared memory key by key and written out as contiguous runs.
constexpr unsigned long long kOrderAggregate = 1ull << 32;   // status word: the tile's own count
constexpr unsigned long long kOrderInclusive = 2ull << 32;   // status word: the count through this tile
constexpr int kOrderWaitLimit = 1 << 22;
constexpr int kOrderLookDepth = 4;   // look-back words per lane and round: 128 predecessors

// exclusive prefix of v over the block's threads (in thread order) and the block's total; every thread calls it
template <class T>
BTE_DI T blockExclusiveScan(T v, T* warpSum, T& total)
{
    const int lane = static_cast<int>(threadIdx.x & 31u), warp = static_cast<int>(threadIdx.x >> 5);
    const int warps = static_cast<int>(blockDim.x >> 5);
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < warps ? warpSum[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warpSum[lane] = w;
    }
    __syncthreads();
    total = warpSum[warps - 1];
    const T excl = x - v + (warp > 0 ? warpSum[warp - 1] : T(0));
    __syncthreads();   // warpSum is reused by the next call
    return excl;
}

__global__ void __launch_bounds__(256, 4) kOrderCompact(DevPaths P, int bounce, int lo, int n, int* out, int stride,
                                                     int compaction)
{
    if (tailTakesOver(P, bounce)) return;
    __shared__ unsigned long long warpSum[32];
    __shared__ int tileSh;
    __shared__ int keyStart[kSortKeys], keyTotal[kSortKeys], keyBase[kSortKeys];
    __shared__ int stage[kOrderTile];
    const int tiles = (P.count + kOrderTile - 1) / kOrderTile;
    unsigned long long* status = P.orderStatus + static_cast<size_t>(compaction) * tiles * kSortKeys;
    if (threadIdx.x == 0) tileSh = atomicAdd(P.orderTicket + compaction, 1);
    __syncthreads();
    const int tile = tileSh;
    // this thread's 32 keys (two 16-byte loads), key e in byte e & 3 of word e >> 2; paths at or beyond count
    // read as ended
    const int first = tile * kOrderTile + static_cast<int>(threadIdx.x) * 32;
    const uint4 kw0 = *reinterpret_cast<const uint4*>(P.pathKey + first);
    const uint4 kw1 = *reinterpret_cast<const uint4*>(P.pathKey + first + 16);
    uint32_t words[8] = {kw0.x, kw0.y, kw0.z, kw0.w, kw1.x, kw1.y, kw1.z, kw1.w};
    if (first + 32 > P.count) {
#pragma unroll
        for (int e = 0; e < 32; ++e)
            if (first + e >= P.count) words[e >> 2] |= 0xffu << (8 * (e & 3));
    }
    // per-key counts of the thread, 16 bits per key: keys lo .. lo+3 in cA, lo+4 .. lo+5 in cB
    unsigned long long cA = 0, cB = 0;
#pragma unroll
    for (int e = 0; e < 32; ++e) {
        const unsigned int d = ((words[e >> 2] >> (8 * (e & 3))) & 0xffu) - static_cast<unsigned int>(lo);
        if (d < static_cast<unsigned int>(n)) {
            if (d < 4u) cA += 1ull << (16 * d);
            else cB += 1ull << (16 * (d - 4u));
        }
    }
    unsigned long long tA, tB = 0;
    const unsigned long long xA = blockExclusiveScan(cA, warpSum, tA);
    unsigned long long xB = 0;
    if (n > 4) xB = blockExclusiveScan(cB, warpSum, tB);
    // per key: this thread's first staging slot, the tile's count and its start in the staging array
    int pos[kSortKeys];
    int run = 0;
#pragma unroll
    for (int j = 0; j < kSortKeys; ++j) {
        const unsigned long long x = j < 4 ? xA : xB, t = j < 4 ? tA : tB;
        const int sh = 16 * (j & 3);
        const int total = j < n ? static_cast<int>((t >> sh) & 0xffffu) : 0;
        pos[j] = run + static_cast<int>((x >> sh) & 0xffffu);
        if (threadIdx.x == 0 && j < n) { keyStart[j] = run; keyTotal[j] = total; }
        run += total;
    }
    __syncthreads();   // keyStart / keyTotal (written by thread 0) before any warp reads them
    // publish, look back, publish the inclusive count: warp j for key j, 128 predecessors per round
    const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31u);
    if (warp < n) {
        const int j = warp;
        volatile unsigned long long* st = status + static_cast<size_t>(tile) * kSortKeys + j;
        const unsigned int own = static_cast<unsigned int>(keyTotal[j]);
        if (lane == 0) *st = (tile == 0 ? kOrderInclusive : kOrderAggregate) | own;
        unsigned int prefix = 0;
        for (int base = tile - 1; base >= 0; base -= 32 * kOrderLookDepth) {
            // predecessor base - (32 q + lane) in word q of this lane; before the first tile: inclusive 0
            unsigned long long w[kOrderLookDepth];
            const volatile unsigned long long* ps[kOrderLookDepth];
            bool wait = false;
#pragma unroll
            for (int q = 0; q < kOrderLookDepth; ++q) {
                const int p = base - 32 * q - lane;
                ps[q] = status + static_cast<size_t>(p < 0 ? 0 : p) * kSortKeys + j;
                w[q] = p >= 0 ? *ps[q] : kOrderInclusive;
                wait |= (w[q] >> 32) == 0ull;
            }
            for (int spins = 0; __any_sync(0xffffffffu, wait); ++spins) {
                if (spins > kOrderWaitLimit) {   // never for a running grid: give up with the error flag
                    if (lane == 0) atomicOr(P.errorFlags, 4u);
#pragma unroll
                    for (int q = 0; q < kOrderLookDepth; ++q) w[q] = kOrderInclusive;
                    break;
                }
                __nanosleep(64);
                wait = false;
#pragma unroll
                for (int q = 0; q < kOrderLookDepth; ++q) {
                    if ((w[q] >> 32) == 0ull) w[q] = *ps[q];
                    wait |= (w[q] >> 32) == 0ull;
                }
            }
            // the nearest inclusive word (smallest 32 q + lane) ends the sum
            bool found = false;
#pragma unroll
            for (int q = 0; q < kOrderLookDepth; ++q) {
                if (found) break;
                const unsigned int inc = __ballot_sync(0xffffffffu, (w[q] >> 32) == 2ull);
                const int stop = inc ? __ffs(inc) - 1 : 31;
                prefix += __reduce_add_sync(0xffffffffu, lane <= stop ? static_cast<unsigned int>(w[q]) : 0u);
                found = inc != 0u;
            }
            if (found) break;
        }
        if (lane == 0) {
            if (tile > 0) *st = kOrderInclusive | (prefix + own);
            keyBase[j] = static_cast<int>(prefix);
            if (tile == tiles - 1) {
                const int total = static_cast<int>(prefix + own);
                if (lo == kKeyNext) P.rayCount[bounce + 1] = total;
                else P.sortCount[bounce * kSortKeys + lo + j] = total;
            }
        }
    }
    // stage the tile's selected paths key by key, in index order
#pragma unroll
    for (int e = 0; e < 32; ++e) {
        const unsigned int d = ((words[e >> 2] >> (8 * (e & 3))) & 0xffu) - static_cast<unsigned int>(lo);
#pragma unroll
        for (int jj = 0; jj < kSortKeys; ++jj)
            if (d == static_cast<unsigned int>(jj) && jj < n) stage[pos[jj]++] = first + e;
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        int* o = out + static_cast<size_t>(j) * stride + keyBase[j];
        const int* src = stage + keyStart[j];
        for (int i = static_cast<int>(threadIdx.x); i < keyTotal[j]; i += static_cast<int>(blockDim.x)) o[i] = src[i];
    }
}

// ---------------------------------------------------------------- connect
// src/wavefront/ray_connect.cu:52-72: occlusion in (1e-4, tMax); an occluded
// slot loses its visibility bit.
template <int Width>
__global__ void __launch_bounds__(256) kConnect(DevScene s, DevPaths P, int bounce)
{
    const int count = P.shadowCount[bounce];
    if (tailTakesOver(P, bounce)) return;
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += stride) {
        const int e = P.shadowQueue[k];
        const int path = e / P.slots;
        const int slot = e - path * P.slots;
        const float4 o = P.shOrigin[path];
        const float4 d = P.shDir[e];
        const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, s.sceneMaxAbs);
        if (traceOccludedW<Width>(s, r, kEps, d.w, P.errorFlags)) atomicAnd(P.shMask + path, ~(1u << slot));
    }
}

// Persistent lanes with ray refill need only ceil(count / 32) warps: those take every ray between them
// (any non-empty subset of warps drains the queue), so the warps above that leave before touching the
// shared fetch counter.  With the few rays of the last bounces this spares thousands of same-address
// atomics per launch.
BTE_DI bool warpNotNeeded(int count)
{
    const long long warp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    return warp * 32 >= count;
}

// ---------------------------------------------------------------- extend / connect over the 8-wide tree
// Same results as kExtend / kConnect, but each lane keeps its walk state
// across iterations and takes a new ray (warp-aggregated fetch from a
// per-bounce counter) as soon as its current one ends, so that lanes do not
// idle until the slowest ray of their warp finishes.
// 64 registers (no spills) keep 8 blocks of 128 threads resident per SM; 72 (7 blocks) measured 1.8% slower per
// frame on the 1080p bench scene
#ifndef BTE_EXTEND_MAXNREG
#define BTE_EXTEND_MAXNREG 64
#endif
template <bool Multi>
__global__ void __maxnreg__(BTE_EXTEND_MAXNREG) kExtendWide(DevScene s, DevPaths P, int bounce)
{
    const int count = P.rayCount[bounce];
    if (tailTakesOver(P, bounce)) return;
    const int* __restrict__ q = raySorted(P, bounce, count) ? P.sortedQueue : P.queue[bounce & 1];
    uint2 stack[kWideStack];
    if (count <= static_cast<int>((gridDim.x * blockDim.x) >> 3)) {   // few rays: eight lanes per ray
        const int g = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
        if (g >= count) return;
        const int idx = q[g];
        const DevScene& ss = sceneOf<Multi>(s, P, idx);
        const float4 o = P.o[idx];
        const float4 d = P.d[idx];
        const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, ss.sceneMaxAbs);
        float t = 0.0f, u = 0.0f, v = 0.0f;
        int tri = -1;
        if (r.valid && ss.triCount > 0) tri = traceWideGroup<false>(ss, r, kEps, 1e30f, stack, P.errorFlags, t, u, v);
        if ((threadIdx.x & 7u) == 0u) {
            P.hit[idx] = tri >= 0 ? make_float4(t, u, v, __int_as_float(tri)) : make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
            if (P.hitLog) P.hitLog[static_cast<size_t>(idx) * P.maxDepth + bounce] = tri;
            bucketPath(ss, P, bounce, idx, tri);
        }
        return;
    }
    if (warpNotNeeded(count)) return;
    int* fetch = P.fetch + bounce;
    WideWalk<false> w;
    int idx = -1;
    while (true) {
        if (idx < 0) {
            const int slot = appendCoalesced(fetch);
            if (slot >= count) break;
            idx = q[slot];
            const DevScene& ss = sceneOf<Multi>(s, P, idx);
            const float4 o = P.o[idx];
            const float4 d = P.d[idx];
            const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, ss.sceneMaxAbs);
            if (!r.valid || ss.triCount <= 0) {
                P.hit[idx] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
                if (P.hitLog) P.hitLog[static_cast<size_t>(idx) * P.maxDepth + bounce] = -1;
                bucketPath(ss, P, bounce, idx, -1);
                idx = -1;
                continue;
            }
            w.start(r, kEps, 1e30f);
        }
        const DevScene& ss = sceneOf<Multi>(s, P, idx);
        if (w.step(ss, stack, P.errorFlags)) {
            const int tri = w.best;
            P.hit[idx] = tri >= 0 ? make_float4(w.bt, w.bu, w.bv, __int_as_float(tri))
                                  : make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
            if (P.hitLog) P.hitLog[static_cast<size_t>(idx) * P.maxDepth + bounce] = tri;
            bucketPath(ss, P, bounce, idx, tri);
            idx = -1;
        }
    }
}

template <bool Multi>
__global__ void __launch_bounds__(256) kConnectWide(DevScene s, DevPaths P, int bounce)
{
    const int count = P.shadowCount[bounce];
    if (tailTakesOver(P, bounce)) return;
    uint2 stack[kWideStack];
    if (count <= static_cast<int>((gridDim.x * blockDim.x) >> 3)) {   // few rays: eight lanes per ray
        const int g = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
        if (g >= count) return;
        const int e = P.shadowQueue[g];
        const int path = e / P.slots;
        const DevScene& ss = sceneOf<Multi>(s, P, path);
        const float4 o = P.shOrigin[path];
        const float4 d = P.shDir[e];
        const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, ss.sceneMaxAbs);
        if (!r.valid || ss.triCount <= 0) return;
        float t, u, v;
        if (traceWideGroup<true>(ss, r, kEps, d.w, stack, P.errorFlags, t, u, v) >= 0 && (threadIdx.x & 7u) == 0u)
            atomicAnd(P.shMask + path, ~(1u << (e - path * P.slots)));
        return;
    }
    if (warpNotNeeded(count)) return;
    int* fetch = P.fetch + (P.maxDepth + 1) + bounce;
    WideWalk<true> w;
    int e = -1;
    while (true) {
        if (e < 0) {
            const int slot = appendCoalesced(fetch);
            if (slot >= count) break;
            e = P.shadowQueue[slot];
            const int path = e / P.slots;
            const DevScene& ss = sceneOf<Multi>(s, P, path);
            const float4 o = P.shOrigin[path];
            const float4 d = P.shDir[e];
            const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, ss.sceneMaxAbs);
            if (!r.valid || ss.triCount <= 0) { e = -1; continue; }
            w.start(r, kEps, d.w);
        }
        if (w.step(sceneOf<Multi>(s, P, e / P.slots), stack, P.errorFlags)) {
            if (w.hit) {
                const int path = e / P.slots;
                atomicAnd(P.shMask + path, ~(1u << (e - path * P.slots)));
            }
            e = -1;
        }
    }
}

// ---------------------------------------------------------------- tail
// Finishes the paths of the first bounce the wavefront left (tailTakesOver): per path, closest hit,
// shading and its shadow rays, bounce after bounce, with the same per-path operations and counters
// as the wavefront stages.
template <int Width, bool Multi>
__global__ void __launch_bounds__(128) kTail(DevScene s, DevPaths P, FrameParams f)
{
    if (P.tailPaths <= 0) return;
    int b0 = -1;
    for (int b = 0; b < P.maxDepth; ++b)
        if (P.rayCount[b] < P.tailPaths) { b0 = b; break; }
    if (b0 < 0) return;
    const int count = P.rayCount[b0];
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= count) return;
    const int idx = P.queue[b0 & 1][slot];
    const DevScene& ss = sceneOf<Multi>(s, P, idx);
    for (int b = b0; b < P.maxDepth; ++b) {
        if (b > b0) atomicAdd(P.rayCount + b, 1);
        const float4 o = P.o[idx];
        const float4 d = P.d[idx];
        const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, ss.sceneMaxAbs);
        float t = 0.0f, u = 0.0f, v = 0.0f;
        const int tri = traceClosestW<Width>(ss, r, kEps, 1e30f, t, u, v, P.errorFlags);
        P.hit[idx] = make_float4(t, u, v, __int_as_float(tri));
        if (P.hitLog) P.hitLog[static_cast<size_t>(idx) * P.maxDepth + b] = tri;
        const bool alive = shadePath(ss, P, f, b, idx, false);
        uint32_t mask = P.shMask[idx];
        if (mask) {
            atomicAdd(P.shadowCount + b, __popc(mask));
            const float4 so = P.shOrigin[idx];
            const size_t base = static_cast<size_t>(idx) * P.slots;
            for (uint32_t m = mask; m; m &= m - 1u) {
                const int sl = __ffs(m) - 1;
                const float4 sd = P.shDir[base + sl];
                const RayPre sr = rayPre(so.x, so.y, so.z, sd.x, sd.y, sd.z, ss.sceneMaxAbs);
                if (traceOccludedW<Width>(ss, sr, kEps, sd.w, P.errorFlags)) mask &= ~(1u << sl);
            }
            P.shMask[idx] = mask;
        }
        if (!alive || b + 1 >= P.maxDepth) break;
    }
}

// kTail over the 8-wide tree with eight lanes per path: a group of eight lanes walks the path's closest-hit and
// shadow rays together (traceWideGroup: the same hits as one lane's walk), lane 0 of the group shades.  Each path
// runs its bounces back to back, so the tail costs the longest remaining path rather than the sum over bounces of
// each bounce's slowest ray (the wavefront's last launches, a few thousand rays each, are latency-bound).
template <bool Multi>
__global__ void __launch_bounds__(128) kTailGroup(DevScene s, DevPaths P, FrameParams f)
{
    if (P.tailPaths <= 0) return;
    int b0 = -1;
    for (int b = 0; b < P.maxDepth; ++b)
        if (P.rayCount[b] < P.tailPaths) { b0 = b; break; }
    if (b0 < 0) return;
    const int count = P.rayCount[b0];
    const int g = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
    if (g >= count) return;   // whole groups: 8 divides the block
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gmask = 0xffu << (lane & ~7u);
    const bool leader = (lane & 7u) == 0u;
    const int idx = P.queue[b0 & 1][g];
    const DevScene& ss = sceneOf<Multi>(s, P, idx);
    uint2 stack[kWideStack];
    for (int b = b0; b < P.maxDepth; ++b) {
        if (b > b0 && leader) atomicAdd(P.rayCount + b, 1);
        const float4 o = P.o[idx];
        const float4 d = P.d[idx];
        const RayPre r = rayPre(o.x, o.y, o.z, d.x, d.y, d.z, ss.sceneMaxAbs);
        float t = 0.0f, u = 0.0f, v = 0.0f;
        const int tri = (r.valid && ss.triCount > 0)
                            ? traceWideGroup<false>(ss, r, kEps, 1e30f, stack, P.errorFlags, t, u, v) : -1;
        int alive = 0;
        if (leader) {
            P.hit[idx] = tri >= 0 ? make_float4(t, u, v, __int_as_float(tri))
                                  : make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
            if (P.hitLog) P.hitLog[static_cast<size_t>(idx) * P.maxDepth + b] = tri;
            alive = shadePath(ss, P, f, b, idx, false) ? 1 : 0;
        }
        __syncwarp(gmask);   // the leader's path state and shadow slots, before the group reads them
        alive = __shfl_sync(gmask, alive, 0, 8);
        uint32_t mask = P.shMask[idx];
        if (mask) {
            if (leader) atomicAdd(P.shadowCount + b, __popc(mask));
            const float4 so = P.shOrigin[idx];
            const size_t base = static_cast<size_t>(idx) * P.slots;
            for (uint32_t m = mask; m; m &= m - 1u) {
                const int sl = __ffs(m) - 1;
                const float4 sd = P.shDir[base + sl];
                const RayPre sr = rayPre(so.x, so.y, so.z, sd.x, sd.y, sd.z, ss.sceneMaxAbs);
                float st, su, sv;
                if (sr.valid && ss.triCount > 0 &&
                    traceWideGroup<true>(ss, sr, kEps, sd.w, stack, P.errorFlags, st, su, sv) >= 0)
                    mask &= ~(1u << sl);
            }
            if (leader) P.shMask[idx] = mask;
        }
        __syncwarp(gmask);
        if (!alive || b + 1 >= P.maxDepth) break;
    }
}

// Adds v to *counter with one atomic per group of lanes that arrive here together with the same key (the
// counter is the same for equal keys); lanes of a warp may be at different bounces in the megakernel.
BTE_DI void groupedAdd(int* counter, int key, int v)
{
    const unsigned active = __activemask();
    const unsigned group = __match_any_sync(active, key);
    const int total = __reduce_add_sync(group, v);
    if (static_cast<unsigned>(__ffs(group) - 1) == (threadIdx.x & 31u) && total != 0) atomicAdd(counter, total);
}

// RenderMode::Megakernel, src/optix_programs.cu:54-108: one thread per pixel and one RNG stream per pixel and
// frame, rngSeed(pixel, frameIndex) = makeRng(hashUint(pixel ^ frameIndex * 0x9e3779b9)), carried through f.spp
// paths in turn, each drawing its jitter first.  Each path runs the tail kernel's bounce loop on the pixel's own
// path slot (the stream returns through P.o.w); the paths' radiance is summed in sample order from zero, scaled
// by div3, folded into the FP32 Welford mean once per frame (n = frames so far + 1) and into the FP64 sum, then
// packed.  With features on (aovAccum), each path's feature albedo and normal (written by shadePath into the
// pixel's slot at the path's first hit that is not a mirror or dielectric) are summed the same way and their per-frame mean folded into aovAccum, so the
// denoiser sees the same features in both render modes.
template <int Width>
__global__ void __launch_bounds__(128) kMegakernel(DevScene s, DevPaths P, FrameParams f, float* accum,
                                                   double* accumD, uint32_t* framebuffer, uint32_t* extFramebuffer,
                                                   float* aovAccum)
{
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    const int wh = f.width * f.height;
    if (pix >= wh || pix >= P.count) return;
    const uint32_t frameIndex = *f.frameIndex;
    const int px = pix % f.width, py = pix / f.width;
    uint32_t rng = rngSeed(static_cast<uint32_t>(pix), frameIndex);
    V3 sum = v3(0.0f, 0.0f, 0.0f);
    float feat[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const bool features = aovAccum && P.aovAlbedo;
    for (int k = 0; k < f.spp; ++k) {
        const float jx = rngNext(rng) - 0.5f;
        const float jy = rngNext(rng) - 0.5f;
        V3 o, d;
        primaryRay(px, py, f.width, f.height, f.cam, f.tanHalf, jx, jy, o, d);
        P.o[pix] = make_float4(o.x, o.y, o.z, __uint_as_float(rng));
        P.d[pix] = make_float4(d.x, d.y, d.z, 1.0f);
        P.tp[pix] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        P.L[pix] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(1u << 16));
        P.shMask[pix] = 0u;
        for (int b = 0; b < P.maxDepth; ++b) {
            groupedAdd(P.rayCount + b, b, 1);
            const float4 ro = P.o[pix];
            const float4 rd = P.d[pix];
            const RayPre r = rayPre(ro.x, ro.y, ro.z, rd.x, rd.y, rd.z, s.sceneMaxAbs);
            float t = 0.0f, u = 0.0f, v = 0.0f;
            const int tri = traceClosestW<Width>(s, r, kEps, 1e30f, t, u, v, P.errorFlags);
            P.hit[pix] = make_float4(t, u, v, __int_as_float(tri));
            const bool alive = shadePath(s, P, f, b, pix, false);
            uint32_t mask = P.shMask[pix];
            groupedAdd(P.shadowCount + b, b, __popc(mask));
            if (mask) {
                const float4 so = P.shOrigin[pix];
                const size_t base = static_cast<size_t>(pix) * P.slots;
                for (uint32_t m = mask; m; m &= m - 1u) {
                    const int sl = __ffs(m) - 1;
                    const float4 sd = P.shDir[base + sl];
                    const RayPre sr = rayPre(so.x, so.y, so.z, sd.x, sd.y, sd.z, s.sceneMaxAbs);
                    if (traceOccludedW<Width>(s, sr, kEps, sd.w, P.errorFlags)) mask &= ~(1u << sl);
                }
                P.shMask[pix] = mask;
            }
            if (!alive || b + 1 >= P.maxDepth) break;
        }
        const float4 L4 = P.L[pix];
        sum = add3(sum, resolveShadows(P, pix, v3(L4.x, L4.y, L4.z)));
        rng = __float_as_uint(P.o[pix].w);
        if (features) {
            const float4 a = P.aovAlbedo[pix], nn = P.aovNormal[pix];
            feat[0] += a.x; feat[1] += a.y; feat[2] += a.z;
            feat[3] += nn.x; feat[4] += nn.y; feat[5] += nn.z;
        }
    }
    if (features) {
        const float paths = static_cast<float>(f.spp);
        const float n = static_cast<float>(frameIndex + 1u);
        for (int c = 0; c < 6; ++c) {
            float m = aovAccum[6 * static_cast<size_t>(pix) + c];
            m = m + (feat[c] / paths - m) / n;
            aovAccum[6 * static_cast<size_t>(pix) + c] = m;
        }
    }
    const V3 c = div3(sum, static_cast<float>(f.spp));
    const float n = static_cast<float>(frameIndex + 1u);
    float ax = accum[3 * pix], ay = accum[3 * pix + 1], az = accum[3 * pix + 2];
    ax = ax + (c.x - ax) / n;
    ay = ay + (c.y - ay) / n;
    az = az + (c.z - az) / n;
    accum[3 * pix] = ax; accum[3 * pix + 1] = ay; accum[3 * pix + 2] = az;
    accumD[3 * pix] += static_cast<double>(c.x);
    accumD[3 * pix + 1] += static_cast<double>(c.y);
    accumD[3 * pix + 2] += static_cast<double>(c.z);
    const uint32_t px32 = packGamma(ax, ay, az);
    framebuffer[pix] = px32;
    if (extFramebuffer) extFramebuffer[pix] = px32;
}

// ---------------------------------------------------------------- present
// src/wavefront/ray_present.cu:43-62 for spp consecutive samples per pixel:
// FP32 Welford mean (rt_path_integrator.cuh:72-87) in sample order, an FP64
// running sum, and the gamma-2.2 RGBA8 pack (:93-105).
__global__ void __launch_bounds__(256) kPresent(DevPaths P, FrameParams f, float* accum, double* accumD,
                                                uint32_t* framebuffer, uint32_t* extFramebuffer, float* aovAccum)
{
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    const int wh = f.width * f.height;
    if (pix >= wh) return;
    const uint32_t frameIndex = *f.frameIndex;
    float ax = accum[3 * pix], ay = accum[3 * pix + 1], az = accum[3 * pix + 2];
    double sx = accumD[3 * pix], sy = accumD[3 * pix + 1], sz = accumD[3 * pix + 2];
    for (int s = 0; s < f.spp; ++s) {
        const int idx = s * wh + pix;
        const float4 L4 = P.L[idx];
        V3 L = resolveShadows(P, idx, v3(L4.x, L4.y, L4.z));
        P.L[idx] = make_float4(L.x, L.y, L.z, L4.w);
        const float n = static_cast<float>(frameIndex + static_cast<uint32_t>(s) + 1u);
        ax = ax + (L.x - ax) / n;
        ay = ay + (L.y - ay) / n;
        az = az + (L.z - az) / n;
        sx += static_cast<double>(L.x);
        sy += static_cast<double>(L.y);
        sz += static_cast<double>(L.z);
    }
    accum[3 * pix] = ax; accum[3 * pix + 1] = ay; accum[3 * pix + 2] = az;
    accumD[3 * pix] = sx; accumD[3 * pix + 1] = sy; accumD[3 * pix + 2] = sz;
    if (aovAccum && P.aovAlbedo) {   // running means of the feature albedo and normal, [W*H][6]
        float m[6];
        for (int c = 0; c < 6; ++c) m[c] = aovAccum[6 * static_cast<size_t>(pix) + c];
        for (int s = 0; s < f.spp; ++s) {
            const int idx = s * wh + pix;
            const float4 a = P.aovAlbedo[idx], nn = P.aovNormal[idx];
            const float x[6] = {a.x, a.y, a.z, nn.x, nn.y, nn.z};
            const float n = static_cast<float>(frameIndex + static_cast<uint32_t>(s) + 1u);
            for (int c = 0; c < 6; ++c) m[c] = m[c] + (x[c] - m[c]) / n;
        }
        for (int c = 0; c < 6; ++c) aovAccum[6 * static_cast<size_t>(pix) + c] = m[c];
    }
    const uint32_t px = packGamma(ax, ay, az);
    framebuffer[pix] = px;
    if (extFramebuffer) extFramebuffer[pix] = px;
}

// present for batched views: one thread per pixel of the frame's pixel space
__global__ void __launch_bounds__(256) kPresentViews(DevPaths P, FrameParams f, int totalPixels)
{
    const int gpix = blockIdx.x * blockDim.x + threadIdx.x;
    if (gpix >= totalPixels) return;
    int v = 0;
    while (v + 1 < f.viewCount && gpix >= f.views[v + 1].pixelOffset) ++v;
    const ViewDesc& vd = f.views[v];
    const int pix = gpix - vd.pixelOffset;
    const int wh = vd.width * vd.height;
    float ax = vd.accum[3 * pix], ay = vd.accum[3 * pix + 1], az = vd.accum[3 * pix + 2];
    double sx = vd.accumD[3 * pix], sy = vd.accumD[3 * pix + 1], sz = vd.accumD[3 * pix + 2];
    for (int s = 0; s < vd.spp; ++s) {
        const int idx = vd.pathOffset + s * wh + pix;
        const float4 L4 = P.L[idx];
        V3 L = resolveShadows(P, idx, v3(L4.x, L4.y, L4.z));
        P.L[idx] = make_float4(L.x, L.y, L.z, L4.w);
        const float n = static_cast<float>(vd.frameIndex + static_cast<uint32_t>(s) + 1u);
        ax = ax + (L.x - ax) / n;
        ay = ay + (L.y - ay) / n;
        az = az + (L.z - az) / n;
        sx += static_cast<double>(L.x);
        sy += static_cast<double>(L.y);
        sz += static_cast<double>(L.z);
    }
    vd.accum[3 * pix] = ax; vd.accum[3 * pix + 1] = ay; vd.accum[3 * pix + 2] = az;
    vd.accumD[3 * pix] = sx; vd.accumD[3 * pix + 1] = sy; vd.accumD[3 * pix + 2] = sz;
    vd.framebuffer[pix] = packGamma(ax, ay, az);
}

// ---------------------------------------------------------------- debug / parity kernels
template <int Width>
__global__ void kTraceClosestRays(DevScene s, const float* rays, int n, int* outTri, float* outTuv, unsigned int* err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r6 = rays + 6 * static_cast<size_t>(i);
    const RayPre r = rayPre(r6[0], r6[1], r6[2], r6[3], r6[4], r6[5], s.sceneMaxAbs);
    float t = 0.0f, u = 0.0f, v = 0.0f;
    const int tri = traceClosestW<Width>(s, r, kEps, 1e30f, t, u, v, err);
    outTri[i] = tri;
    outTuv[3 * i] = t; outTuv[3 * i + 1] = u; outTuv[3 * i + 2] = v;
}

template <int Width>
__global__ void kTraceOccludedRays(DevScene s, const float* rays, const float* tmax, int n, uint8_t* out, unsigned int* err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r6 = rays + 6 * static_cast<size_t>(i);
    const RayPre r = rayPre(r6[0], r6[1], r6[2], r6[3], r6[4], r6[5], s.sceneMaxAbs);
    out[i] = traceOccludedW<Width>(s, r, kEps, tmax[i], err) ? 1 : 0;
}

// the same queries through the 8-lanes-per-ray walk (8-wide tree): ray i is walked by lanes 8i .. 8i+7
__global__ void kTraceClosestRaysGroup(DevScene s, const float* rays, int n, int* outTri, float* outTuv, unsigned int* err)
{
    const int i = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
    if (i >= n) return;
    const float* r6 = rays + 6 * static_cast<size_t>(i);
    const RayPre r = rayPre(r6[0], r6[1], r6[2], r6[3], r6[4], r6[5], s.sceneMaxAbs);
    float t = 0.0f, u = 0.0f, v = 0.0f;
    uint2 stack[kWideStack];
    const int tri = (r.valid && s.triCount > 0) ? traceWideGroup<false>(s, r, kEps, 1e30f, stack, err, t, u, v) : -1;
    if ((threadIdx.x & 7u) == 0u) {
        outTri[i] = tri;
        outTuv[3 * i] = t; outTuv[3 * i + 1] = u; outTuv[3 * i + 2] = v;
    }
}

__global__ void kTraceOccludedRaysGroup(DevScene s, const float* rays, const float* tmax, int n, uint8_t* out,
                                        unsigned int* err)
{
    const int i = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
    if (i >= n) return;
    const float* r6 = rays + 6 * static_cast<size_t>(i);
    const RayPre r = rayPre(r6[0], r6[1], r6[2], r6[3], r6[4], r6[5], s.sceneMaxAbs);
    float t, u, v;
    uint2 stack[kWideStack];
    const bool occ = r.valid && s.triCount > 0 && traceWideGroup<true>(s, r, kEps, tmax[i], stack, err, t, u, v) >= 0;
    if ((threadIdx.x & 7u) == 0u) out[i] = occ ? 1 : 0;
}

__global__ void kEnvQuery(DevScene s, int op, const float* in, int n, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (op == 0) {
        const V3 r = envEval(s.env, v3(in[3 * i], in[3 * i + 1], in[3 * i + 2]));
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    } else if (op == 1) {
        out[i] = envPdf(s.env, v3(in[3 * i], in[3 * i + 1], in[3 * i + 2]));
    } else {
        const EnvSample e = envSample(s.env, in[2 * i], in[2 * i + 1]);
        float* o = out + 7 * static_cast<size_t>(i);
        o[0] = e.dir.x; o[1] = e.dir.y; o[2] = e.dir.z; o[3] = e.pdf; o[4] = e.rad.x; o[5] = e.rad.y; o[6] = e.rad.z;
    }
}

__global__ void kMathEval(int fn, const float* a, const float* b, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r;
    switch (fn) {
    case 0: r = m::sinf_(a[i]); break;
    case 1: r = m::cosf_(a[i]); break;
    case 2: r = m::tanf_(a[i]); break;
    case 3: r = m::expf_(a[i]); break;
    case 4: r = m::logf_(a[i]); break;
    case 5: r = m::powf_(a[i], b[i]); break;
    case 6: r = m::atan2f_(a[i], b[i]); break;
    case 7: r = m::acosf_(a[i]); break;
    // CUDA's own functions, for the accuracy comparison of the deterministic set
    case 100: r = sinf(a[i]); break;
    case 101: r = cosf(a[i]); break;
    case 102: r = tanf(a[i]); break;
    case 103: r = expf(a[i]); break;
    case 104: r = logf(a[i]); break;
    case 105: r = powf(a[i], b[i]); break;
    case 106: r = atan2f(a[i], b[i]); break;
    case 107: r = acosf(a[i]); break;
    default: r = NAN; break;
    }
    out[i] = r;
}

// op 0: eval(wi, wo) -> 3; op 1: pdf(wi, wo) -> 1; op 2: sample(wi, u[3]) -> wo 3, weight 3, pdf 1, eta 1
__global__ void kBsdfQuery(BsdfData g, int op, const float* wi, const float* x, int n, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Bsdf b;
    b.type = g.type;
    b.p0 = make_float4(g.p0.x, g.p0.y, g.p0.z, g.p0.w);
    b.p1 = make_float4(g.p1.x, g.p1.y, g.p1.z, g.p1.w);
    b.p2 = make_float4(g.p2.x, g.p2.y, g.p2.z, g.p2.w);
    b.p3 = make_float4(g.p3.x, g.p3.y, g.p3.z, g.p3.w);
    BRec r = brec0();
    r.wi = v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    if (op == 0 || op == 1) {
        r.wo = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        r.measure = kSolid;
        if (op == 0) {
            const V3 v = bsdfEval(b, r);
            out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
        } else {
            out[i] = bsdfPdf(b, r);
        }
    } else {
        r.rndExtra = x[3 * i];
        const V3 w = bsdfSample(b, r, x[3 * i + 1], x[3 * i + 2]);
        float* o = out + 8 * static_cast<size_t>(i);
        o[0] = r.wo.x; o[1] = r.wo.y; o[2] = r.wo.z;
        o[3] = w.x; o[4] = w.y; o[5] = w.z;
        o[6] = bsdfPdf(b, r);
        o[7] = r.eta;
    }
}

__global__ void kTexCompare(cudaTextureObject_t tex, const float4* texels, int w, int h, int wrapV, const float* uv, int n,
                            float* outHw, float* outSw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float u = uv[2 * i], v = uv[2 * i + 1];
    const float4 a = tex2D<float4>(tex, u, v);
    const float4 b = texFloat4(texels, w, h, wrapV != 0, u, v);
    outHw[4 * i] = a.x; outHw[4 * i + 1] = a.y; outHw[4 * i + 2] = a.z; outHw[4 * i + 3] = a.w;
    outSw[4 * i] = b.x; outSw[4 * i + 1] = b.y; outSw[4 * i + 2] = b.z; outSw[4 * i + 3] = b.w;
}

// ---------------------------------------------------------------- launchers
void launchGenerate(const DevPaths& P, const FrameParams& f, cudaStream_t st)
{
    const int blocks = (P.count + 255) / 256;
    kGenerate<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(P, f);
}
void launchRaySort(const DevPaths& P, int bounce, int grid, cudaStream_t st)
{
    kRayBins<<<1, 1024, 0, st>>>(P, bounce);
    kRayScatter<<<grid, 256, 0, st>>>(P, bounce);
}
int orderTiles(int paths) { return (paths + kOrderTile - 1) / kOrderTile; }
// compaction 2b builds bounce b's buckets, 2b+1 the queue of bounce b+1 (each has its own ticket and status words)
void launchOrder(const DevPaths& P, int bounce, bool nextQueue, cudaStream_t st)
{
    const int lo = nextQueue ? kKeyNext : 0, n = nextQueue ? 1 : kSortKeys;
    int* out = nextQueue ? P.queue[(bounce + 1) & 1] : P.sortQueue;
    const int stride = nextQueue ? 0 : P.count;
    kOrderCompact<<<orderTiles(P.count), 256, 0, st>>>(P, bounce, lo, n, out, stride, 2 * bounce + (nextQueue ? 1 : 0));
}
// Frames over several scenes (P.scenes) run the stage kernels' multi-scene instances; those scenes all use the
// 8-wide tree (checked by the host).
void launchExtend(const DevScene& s, const DevPaths& P, int bounce, int grid, int block, cudaStream_t st)
{
    if (P.scenes) kExtendWide<true><<<grid, block, 0, st>>>(s, P, bounce);
    else if (s.bvhWidth == 8) kExtendWide<false><<<grid, block, 0, st>>>(s, P, bounce);
    else kExtend<2><<<grid, block, 0, st>>>(s, P, bounce);
}
void launchShade(const DevScene& s, const DevPaths& P, const FrameParams& f, int bounce, int grid, int block,
                 int minBlocks, cudaStream_t st)
{
    if (P.scenes) {
        if (minBlocks == 4) kShade<4, true><<<grid, block, 0, st>>>(s, P, f, bounce);
        else if (minBlocks == 3) kShade<3, true><<<grid, block, 0, st>>>(s, P, f, bounce);
        else kShade<2, true><<<grid, block, 0, st>>>(s, P, f, bounce);
        return;
    }
    if (minBlocks == 4) kShade<4, false><<<grid, block, 0, st>>>(s, P, f, bounce);
    else if (minBlocks == 3) kShade<3, false><<<grid, block, 0, st>>>(s, P, f, bounce);
    else kShade<2, false><<<grid, block, 0, st>>>(s, P, f, bounce);
}
void launchConnect(const DevScene& s, const DevPaths& P, int bounce, int grid, int block, cudaStream_t st)
{
    if (P.scenes) kConnectWide<true><<<grid, block, 0, st>>>(s, P, bounce);
    else if (s.bvhWidth == 8) kConnectWide<false><<<grid, block, 0, st>>>(s, P, bounce);
    else kConnect<2><<<grid, block, 0, st>>>(s, P, bounce);
}
void launchPresentViews(const DevPaths& P, const FrameParams& f, int totalPixels, cudaStream_t st)
{
    kPresentViews<<<(totalPixels + 255) / 256, 256, 0, st>>>(P, f, totalPixels);
}
void launchTail(const DevScene& s, const DevPaths& P, const FrameParams& f, cudaStream_t st)
{
    if (P.tailPaths <= 0) return;
    const int n = P.tailPaths < P.count ? P.tailPaths : P.count;
    const int blocks = (n + 127) / 128;
    const int groupBlocks = static_cast<int>((8LL * n + 127) / 128);   // eight lanes per path
    if (P.scenes) kTailGroup<true><<<groupBlocks, 128, 0, st>>>(s, P, f);
    else if (s.bvhWidth == 8) kTailGroup<false><<<groupBlocks, 128, 0, st>>>(s, P, f);
    else kTail<2, false><<<blocks, 128, 0, st>>>(s, P, f);
}
void launchMegakernel(const DevScene& s, const DevPaths& P, const FrameParams& f, float* accum, double* accumD,
                      uint32_t* fb, uint32_t* extFb, float* aovAccum, cudaStream_t st)
{
    const int wh = f.width * f.height;
    if (s.bvhWidth == 8) kMegakernel<8><<<(wh + 127) / 128, 128, 0, st>>>(s, P, f, accum, accumD, fb, extFb, aovAccum);
    else kMegakernel<2><<<(wh + 127) / 128, 128, 0, st>>>(s, P, f, accum, accumD, fb, extFb, aovAccum);
}
void launchPresent(const DevPaths& P, const FrameParams& f, float* accum, double* accumD, uint32_t* fb, uint32_t* extFb,
                   float* aovAccum, cudaStream_t st)
{
    const int wh = f.width * f.height;
    kPresent<<<(wh + 255) / 256, 256, 0, st>>>(P, f, accum, accumD, fb, extFb, aovAccum);
}
// gamma-packed RGBA8 of an RGB float image (the denoised frame)
__global__ void kPackImage(const float* __restrict__ rgb, int n, uint32_t* fb, uint32_t* extFb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t px = packGamma(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
    fb[i] = px;
    if (extFb) extFb[i] = px;
}
void launchPackImage(const float* rgb, int n, uint32_t* fb, uint32_t* extFb, cudaStream_t st)
{
    kPackImage<<<(n + 255) / 256, 256, 0, st>>>(rgb, n, fb, extFb);
}
void launchTraceClosestRays(const DevScene& s, const float* rays, int n, int* outTri, float* outTuv, unsigned int* err,
                            int lanes, cudaStream_t st)
{
    if (lanes == 8) kTraceClosestRaysGroup<<<(n + 15) / 16, 128, 0, st>>>(s, rays, n, outTri, outTuv, err);
    else if (s.bvhWidth == 8) kTraceClosestRays<8><<<(n + 127) / 128, 128, 0, st>>>(s, rays, n, outTri, outTuv, err);
    else kTraceClosestRays<2><<<(n + 127) / 128, 128, 0, st>>>(s, rays, n, outTri, outTuv, err);
}
void launchTraceOccludedRays(const DevScene& s, const float* rays, const float* tmax, int n, uint8_t* out, unsigned int* err,
                             int lanes, cudaStream_t st)
{
    if (lanes == 8) kTraceOccludedRaysGroup<<<(n + 15) / 16, 128, 0, st>>>(s, rays, tmax, n, out, err);
    else if (s.bvhWidth == 8) kTraceOccludedRays<8><<<(n + 127) / 128, 128, 0, st>>>(s, rays, tmax, n, out, err);
    else kTraceOccludedRays<2><<<(n + 127) / 128, 128, 0, st>>>(s, rays, tmax, n, out, err);
}
void launchEnvQuery(const DevScene& s, int op, const float* in, int n, float* out, cudaStream_t st)
{
    kEnvQuery<<<(n + 127) / 128, 128, 0, st>>>(s, op, in, n, out);
}
void launchMathEval(int fn, const float* a, const float* b, float* out, int n, cudaStream_t st)
{
    kMathEval<<<(n + 255) / 256, 256, 0, st>>>(fn, a, b, out, n);
}
void launchBsdfQuery(const BsdfData& g, int op, const float* wi, const float* x, int n, float* out, cudaStream_t st)
{
    kBsdfQuery<<<(n + 127) / 128, 128, 0, st>>>(g, op, wi, x, n, out);
}
void launchTexCompare(cudaTextureObject_t tex, const float4* texels, int w, int h, int wrapV, const float* uv, int n,
                      float* outHw, float* outSw, cudaStream_t st)
{
    kTexCompare<<<(n + 127) / 128, 128, 0, st>>>(tex, texels, w, h, wrapV, uv, n, outHw, outSw);
}

int occupancyGrid(int which, int block)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn = which == 0 ? reinterpret_cast<const void*>(kExtend<2>)
                   : which == 1 ? reinterpret_cast<const void*>(kShade<2, false>)
                   : which == 3 ? reinterpret_cast<const void*>(kShade<3, false>)
                   : which == 6 ? reinterpret_cast<const void*>(kShade<4, false>)
                   : which == 4 ? reinterpret_cast<const void*>(kExtendWide<false>)
                   : which == 5 ? reinterpret_cast<const void*>(kConnectWide<false>)
                                : reinterpret_cast<const void*>(kConnect<2>);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, 0) != cudaSuccess || per < 1) per = 1;
    return sms * per;
}

}  // namespace bte
