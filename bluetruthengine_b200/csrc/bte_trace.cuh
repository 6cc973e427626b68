// bte_trace.cuh -- ray traversal: watertight ray/triangle test, BVH2 and 8-wide walks.
//
// Replaces the OptiX calls of the reference (rt_optix_shading.cuh:57-95,
// closest hit in [1e-4, 1e30] and first-hit occlusion in [1e-4, tMax]) with
// software traversal on the SMs.  Closest hit is defined as the smallest t
// of the watertight test of Woop, Benthin and Wald (JCGT 2013) over all
// triangles, ties broken towards the lower triangle index, so the result does
// not depend on the tree or on traversal order.  The box test is the robust
// slab test (tmax scaled by 1 + 2*gamma_3, Ize 2013) and nodes are culled only
// when their entry distance exceeds the current best by a relative margin, so
// culling never changes which triangle wins.  Because the watertight test's t
// carries an absolute error that grows with the coordinates' magnitude
// (cancellation between vertex and origin coordinates), every slab is widened
// by kTriErrK * 2^-24 * (max|origin| + max|scene coordinate|): a node is
// culled only if no triangle inside could report a t the test would accept.
// Barycentrics follow the OptiX convention: u weights v1, v weights v2.
#pragma once

#include "bte_types.cuh"

namespace bte {

struct RayPre {
    float ox, oy, oz;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    float ix, iy, iz;     // reciprocal direction for the slab test (zeros replaced by +-1e-30)
    float px, py, pz;     // per-slab widening in t units
    float nx, ny, nz;     // -origin * reciprocal direction (slab test in fused form)
    bool valid;
};

constexpr float kTriErrK = 96.0f;

BTE_DI float comp3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

BTE_DI RayPre rayPre(float ox, float oy, float oz, float dx, float dy, float dz, float sceneMaxAbs)
{
    RayPre r;
    r.ox = ox; r.oy = oy; r.oz = oz;
    const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    int kz = 0;
    if (ay > ax) kz = 1;
    if (az > (kz == 0 ? ax : ay)) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const float dk = comp3(dx, dy, dz, kz);
    if (dk < 0.0f) { const int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.valid = (dk != 0.0f) && (dk == dk);
    r.Sx = comp3(dx, dy, dz, kx) / dk;
    r.Sy = comp3(dx, dy, dz, ky) / dk;
    r.Sz = 1.0f / dk;
    r.ix = 1.0f / (fabsf(dx) > 1e-30f ? dx : copysignf(1e-30f, dx));
    r.iy = 1.0f / (fabsf(dy) > 1e-30f ? dy : copysignf(1e-30f, dy));
    r.iz = 1.0f / (fabsf(dz) > 1e-30f ? dz : copysignf(1e-30f, dz));
    const float pad = kTriErrK * 5.9604645e-8f * (fmaxf(fabsf(ox), fmaxf(fabsf(oy), fabsf(oz))) + sceneMaxAbs);
    r.px = pad * fabsf(r.ix);
    r.py = pad * fabsf(r.iy);
    r.pz = pad * fabsf(r.iz);
    r.nx = -ox * r.ix;
    r.ny = -oy * r.iy;
    r.nz = -oz * r.iz;
    return r;
}

// Watertight test; returns true with t in [tmin, tmax].  Every product and difference is an explicitly rounded
// operation (__fmul_rn / __fsub_rn / __fadd_rn, and __dmul_rn / __dsub_rn in the double fallback), so no build
// contracts them into fused multiply-adds: hits are identical whether or not the library allows contraction.
BTE_DI float mulSub(float a, float b, float c, float d) { return __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d)); }
BTE_DI float mulSubD(float a, float b, float c, float d)
{
    return static_cast<float>(__dsub_rn(__dmul_rn(static_cast<double>(a), static_cast<double>(b)),
                                        __dmul_rn(static_cast<double>(c), static_cast<double>(d))));
}
BTE_DI bool isectTri(const RayPre& r, float4 a, float4 b, float4 c, float tmin, float tmax, float& ot, float& ou,
                     float& ov)
{
    const float Ax0 = a.x - r.ox, Ay0 = a.y - r.oy, Az0 = a.z - r.oz;
    const float Bx0 = b.x - r.ox, By0 = b.y - r.oy, Bz0 = b.z - r.oz;
    const float Cx0 = c.x - r.ox, Cy0 = c.y - r.oy, Cz0 = c.z - r.oz;
    const float Akz = comp3(Ax0, Ay0, Az0, r.kz), Bkz = comp3(Bx0, By0, Bz0, r.kz), Ckz = comp3(Cx0, Cy0, Cz0, r.kz);
    const float Ax = __fsub_rn(comp3(Ax0, Ay0, Az0, r.kx), __fmul_rn(r.Sx, Akz));
    const float Ay = __fsub_rn(comp3(Ax0, Ay0, Az0, r.ky), __fmul_rn(r.Sy, Akz));
    const float Bx = __fsub_rn(comp3(Bx0, By0, Bz0, r.kx), __fmul_rn(r.Sx, Bkz));
    const float By = __fsub_rn(comp3(Bx0, By0, Bz0, r.ky), __fmul_rn(r.Sy, Bkz));
    const float Cx = __fsub_rn(comp3(Cx0, Cy0, Cz0, r.kx), __fmul_rn(r.Sx, Ckz));
    const float Cy = __fsub_rn(comp3(Cx0, Cy0, Cz0, r.ky), __fmul_rn(r.Sy, Ckz));
    float U = mulSub(Cx, By, Cy, Bx);
    float V = mulSub(Ax, Cy, Ay, Cx);
    float W = mulSub(Bx, Ay, By, Ax);
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = mulSubD(Cx, By, Cy, Bx);
        V = mulSubD(Ax, Cy, Ay, Cx);
        W = mulSubD(Bx, Ay, By, Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float t = __fdiv_rn(T, det);
    if (!(t >= tmin && t <= tmax)) return false;
    ot = t;
    ou = __fdiv_rn(V, det);
    ov = __fdiv_rn(W, det);
    return true;
}

constexpr float kBoxGrow = 1.0f + 2.0f * (3.0f * 5.9604645e-8f) / (1.0f - 3.0f * 5.9604645e-8f);   // 1 + 2*gamma_3
constexpr float kCullMargin = 1.0001f;

// slab test of one child box; returns entry distance in tEnter
BTE_DI bool boxHit(const RayPre& r, float lx, float hx, float ly, float hy, float lz, float hz, float tmin, float tmax,
                   float& tEnter)
{
    const float tx0 = __fmaf_rn(lx, r.ix, r.nx), tx1 = __fmaf_rn(hx, r.ix, r.nx);
    const float ty0 = __fmaf_rn(ly, r.iy, r.ny), ty1 = __fmaf_rn(hy, r.iy, r.ny);
    const float tz0 = __fmaf_rn(lz, r.iz, r.nz), tz1 = __fmaf_rn(hz, r.iz, r.nz);
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1) - r.px, fminf(ty0, ty1) - r.py), fmaxf(fminf(tz0, tz1) - r.pz, tmin));
    const float tf = fminf(fminf(fmaxf(tx0, tx1) + r.px, fmaxf(ty0, ty1) + r.py), fminf(fmaxf(tz0, tz1) + r.pz, tmax)) * kBoxGrow;
    tEnter = tn;
    return tn <= tf;
}

BTE_DI int leafStart(int c) { return (~c) & kLeafStartMask; }
BTE_DI int leafCount(int c) { return ((~c) >> kLeafCountShift) + 1; }

// Closest hit.  Returns the triangle index (original numbering) or -1.
BTE_DI int traceClosest(const DevScene& s, const RayPre& r, float tmin, float tmax, float& tOut, float& uOut,
                        float& vOut, unsigned int* errorFlags)
{
    if (!r.valid || s.triCount <= 0) return -1;
    int best = -1;
    float bt = tmax, bu = 0.0f, bv = 0.0f;
    int stack[kTraversalStack];
    int sp = 0;
    int node = s.rootIsLeaf ? s.rootCode : 0;
    while (true) {
        if (node >= 0) {
            const BvhNode* n = s.nodes + node;
            const float4 lxy = __ldg(&n->lxy), rxy = __ldg(&n->rxy), z = __ldg(&n->z);
            const int4 ch = __ldg(&n->child);
            const float cull = bt * kCullMargin;
            float t0, t1;
            const bool h0 = boxHit(r, lxy.x, lxy.y, lxy.z, lxy.w, z.x, z.y, tmin, cull, t0);
            const bool h1 = boxHit(r, rxy.x, rxy.y, rxy.z, rxy.w, z.z, z.w, tmin, cull, t1);
            if (h0 && h1) {
                int nearC = ch.x, farC = ch.y;
                if (t1 < t0) { nearC = ch.y; farC = ch.x; }
                if (sp < kTraversalStack) stack[sp++] = farC;
                else if (errorFlags) atomicOr(errorFlags, 1u);
                node = nearC;
                continue;
            }
            if (h0) { node = ch.x; continue; }
            if (h1) { node = ch.y; continue; }
        } else {
            const int start = leafStart(node), cnt = leafCount(node);
            for (int k = start; k < start + cnt; ++k) {
                const float4 a = __ldg(s.leafTris + 3 * k);
                const float4 b = __ldg(s.leafTris + 3 * k + 1);
                const float4 c = __ldg(s.leafTris + 3 * k + 2);
                float t, u, v;
                if (isectTri(r, a, b, c, tmin, bt, t, u, v)) {
                    const int idx = __float_as_int(a.w);
                    if (best < 0 || t < bt || (t == bt && idx < best)) { best = idx; bt = t; bu = u; bv = v; }
                }
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    if (best >= 0) { tOut = bt; uOut = bu; vOut = bv; }
    return best;
}

// Any hit in [tmin, tmax].
BTE_DI bool traceOccluded(const DevScene& s, const RayPre& r, float tmin, float tmax, unsigned int* errorFlags)
{
    if (!r.valid || s.triCount <= 0) return false;
    int stack[kTraversalStack];
    int sp = 0;
    int node = s.rootIsLeaf ? s.rootCode : 0;
    const float cull = tmax * kCullMargin;
    while (true) {
        if (node >= 0) {
            const BvhNode* n = s.nodes + node;
            const float4 lxy = __ldg(&n->lxy), rxy = __ldg(&n->rxy), z = __ldg(&n->z);
            const int4 ch = __ldg(&n->child);
            float t0, t1;
            const bool h0 = boxHit(r, lxy.x, lxy.y, lxy.z, lxy.w, z.x, z.y, tmin, cull, t0);
            const bool h1 = boxHit(r, rxy.x, rxy.y, rxy.z, rxy.w, z.z, z.w, tmin, cull, t1);
            if (h0 && h1) {
                int nearC = ch.x, farC = ch.y;
                if (t1 < t0) { nearC = ch.y; farC = ch.x; }
                if (sp < kTraversalStack) stack[sp++] = farC;
                else if (errorFlags) atomicOr(errorFlags, 1u);
                node = nearC;
                continue;
            }
            if (h0) { node = ch.x; continue; }
            if (h1) { node = ch.y; continue; }
        } else {
            const int start = leafStart(node), cnt = leafCount(node);
            for (int k = start; k < start + cnt; ++k) {
                const float4 a = __ldg(s.leafTris + 3 * k);
                const float4 b = __ldg(s.leafTris + 3 * k + 1);
                const float4 c = __ldg(s.leafTris + 3 * k + 2);
                float t, u, v;
                if (isectTri(r, a, b, c, tmin, tmax, t, u, v)) return true;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return false;
}

// ---------------------------------------------------------------- 8-wide traversal
// One ray per thread over WideNode.  A node fetch tests all eight child boxes
// (decoded exactly as the build decoded them, then the same robust slab test
// as above), giving a mask of internal children to visit, keyed by
// slot ^ octant so that the lowest set bit is the child nearest the ray's
// origin side, and a mask of the node's leaf triangles to test.  The stack
// holds (childBase, remaining keys << 8 | imask) groups and deferred leaf
// groups (triBase, kTriGroup | mask): when few lanes of a warp have leaf
// tests, they are pushed and run later with more lanes (the postponing of
// Ylitie, Karras and Laine, HPG 2017).
BTE_DI float wideScale(uint32_t e) { return __uint_as_float(e << 23); }
// byte (selected by `sel` from x) as a float: 0x4b0000qq is 2^23 + q exactly
constexpr uint32_t kTriGroup = 0x80000000u;   // stack entry holds (triBase, leaf-test mask)

// three-input max / min (one instruction on sm_100); NaN operands are ignored, as by fmaxf / fminf chains
BTE_DI float max3f(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
BTE_DI float min3f(float a, float b, float c)
{
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

BTE_DI float byteToFloat(uint32_t x, uint32_t sel)
{
    return __uint_as_float(__byte_perm(x, 0x4b000000u, sel)) - 8388608.0f;
}

// The walk's state, advanced one iteration at a time so that a kernel can
// give a lane a new ray as soon as its current one ends.
template <bool AnyHit>
struct WideWalk {
    RayPre r;
    int sp, visits, best;
    uint32_t oct, nBase, nBits, tBase, tHits;
    float tmin, tmax, bt, bu, bv;
    bool hit;   // any-hit result

    BTE_DI void start(const RayPre& ray, float t0, float t1)
    {
        r = ray;
        tmin = t0; tmax = t1;
        oct = (r.ix < 0.0f ? 1u : 0u) | (r.iy < 0.0f ? 2u : 0u) | (r.iz < 0.0f ? 4u : 0u);
        sp = 0; visits = 0; best = -1;
        bt = t1; bu = 0.0f; bv = 0.0f;
        nBase = 0; nBits = ((1u << oct) << 8) | 1u;     // the root as the only child of a virtual parent
        tBase = 0; tHits = 0;
        hit = false;
    }

    // One iteration: at most one node fetch, then that node's (or a deferred
    // group's) leaf tests, then a pop.  Returns true when the walk has ended.
    // `stack` is the lane's kWideStack-entry array (kept outside the struct
    // so that the scalar state stays in registers).
    BTE_DI bool step(const DevScene& s, uint2* stack, unsigned int* errorFlags)
    {
        if (tHits == 0u && (nBits >> 8)) {
            const uint32_t hits = nBits >> 8;
            const uint32_t key = static_cast<uint32_t>(__ffs(hits) - 1);
            const uint32_t rest = hits & (hits - 1u);
            const uint32_t slot = key ^ oct;
            const uint32_t imaskP = nBits & 0xffu;
            const int child = static_cast<int>(nBase) + __popc(imaskP & ((1u << slot) - 1u));
            if (child < 0 || child >= s.wideNodeCount || ++visits > s.wideNodeCount) {   // never true for a built tree
                if (errorFlags) atomicOr(errorFlags, 2u);
                return true;
            }
            if (rest) {
                if (sp < kWideStack) stack[sp++] = make_uint2(nBase, (rest << 8) | imaskP);
                else if (errorFlags) atomicOr(errorFlags, 1u);
            }
            const float4* np = reinterpret_cast<const float4*>(s.wnodes) + 5 * static_cast<size_t>(child);
            const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2), f3 = __ldg(np + 3), f4 = __ldg(np + 4);
            const uint32_t em = __float_as_uint(f0.w);
            const uint32_t imask = em >> 24;
            // Child plane distance t = (p + q * 2^e - o) / d evaluated as fma(q, 2^e / d, (p - o) / d): the
            // power-of-two product is exact, and the two remaining roundings are covered by the per-ray slab
            // widening (|p + q 2^e| stays within a small multiple of the scene extent).
            const float ax = wideScale(em & 0xffu) * r.ix, ay = wideScale((em >> 8) & 0xffu) * r.iy,
                        az = wideScale((em >> 16) & 0xffu) * r.iz;
            const float cx = (f0.x - r.ox) * r.ix, cy = (f0.y - r.oy) * r.iy, cz = (f0.z - r.oz) * r.iz;
            // slab widening folded into the offsets (its rounding is far inside the widening's margin)
            const float cnx = cx - r.px, cfx = cx + r.px, cny = cy - r.py, cfy = cy + r.py, cnz = cz - r.pz,
                        cfz = cz + r.pz;
            const uint32_t meta[2] = {__float_as_uint(f1.z), __float_as_uint(f1.w)};
            // near plane = low side where the direction is positive, high side where it is negative
            const bool sxn = oct & 1u, syn = oct & 2u, szn = oct & 4u;
            const uint32_t nx[2] = {__float_as_uint(sxn ? f3.z : f2.x), __float_as_uint(sxn ? f3.w : f2.y)};
            const uint32_t fx[2] = {__float_as_uint(sxn ? f2.x : f3.z), __float_as_uint(sxn ? f2.y : f3.w)};
            const uint32_t ny[2] = {__float_as_uint(syn ? f4.x : f2.z), __float_as_uint(syn ? f4.y : f2.w)};
            const uint32_t fy[2] = {__float_as_uint(syn ? f2.z : f4.x), __float_as_uint(syn ? f2.w : f4.y)};
            const uint32_t nz[2] = {__float_as_uint(szn ? f4.z : f3.x), __float_as_uint(szn ? f4.w : f3.y)};
            const uint32_t fz[2] = {__float_as_uint(szn ? f3.x : f4.z), __float_as_uint(szn ? f3.y : f4.w)};
            const float cull = AnyHit ? tmax * kCullMargin : bt * kCullMargin;
            uint32_t hitBits = 0;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int w = c >> 2;
                const uint32_t sel = static_cast<uint32_t>(c & 3) | 0x7440u;   // byte c, two zero bytes, 0x4b
                // (empty slots are inverted boxes; one that still passes has no triangles and no child)
                const float tnx = __fmaf_rn(byteToFloat(nx[w], sel), ax, cnx);
                const float tfx = __fmaf_rn(byteToFloat(fx[w], sel), ax, cfx);
                const float tny = __fmaf_rn(byteToFloat(ny[w], sel), ay, cny);
                const float tfy = __fmaf_rn(byteToFloat(fy[w], sel), ay, cfy);
                const float tnz = __fmaf_rn(byteToFloat(nz[w], sel), az, cnz);
                const float tfz = __fmaf_rn(byteToFloat(fz[w], sel), az, cfz);
                const float tn = max3f(tnx, tny, fmaxf(tnz, tmin));
                const float tf = min3f(tfx, tfy, fminf(tfz, cull)) * kBoxGrow;
                hitBits |= (tn <= tf ? 1u : 0u) << c;
            }
            // internal children that were hit, re-keyed to slot ^ octant (bit c -> bit c ^ oct)
            uint32_t newHits = hitBits & imask;
            if (oct & 1u) newHits = ((newHits & 0x55u) << 1) | ((newHits >> 1) & 0x55u);
            if (oct & 2u) newHits = ((newHits & 0x33u) << 2) | ((newHits >> 2) & 0x33u);
            if (oct & 4u) newHits = ((newHits & 0x0fu) << 4) | ((newHits >> 4) & 0x0fu);
            // triangles of the leaf slots that were hit
            uint32_t triMask = 0;
            for (uint32_t lh = hitBits & ~imask; lh; lh &= lh - 1u) {
                const int c = __ffs(lh) - 1;
                const uint32_t mb = (((c & 4) ? meta[1] : meta[0]) >> (8 * (c & 3))) & 0xffu;
                triMask |= ((1u << (mb >> 5)) - 1u) << (mb & 31u);
            }
            nBase = static_cast<uint32_t>(__float_as_int(f1.x));
            nBits = (newHits << 8) | imask;
            tBase = static_cast<uint32_t>(__float_as_int(f1.y));
            tHits = triMask;
        }
        {   // defer this node's leaf tests while few lanes of the warp have any (more will join later)
            const uint32_t conv = __activemask();
            const uint32_t want = __ballot_sync(conv, tHits != 0u);
            if (tHits != 0u && (nBits >> 8) != 0u && sp < kWideStack &&
                100u * static_cast<uint32_t>(__popc(want)) < static_cast<uint32_t>(s.postponePct * __popc(conv))) {
                stack[sp++] = make_uint2(tBase, kTriGroup | tHits);
                tHits = 0;
            }
        }
        // leaf tests: all of them, or at most s.leafTestsPerStep per step (the rest wait for the next steps,
        // which fetch no node until they are done), so that lanes with many triangles hold the warp less long
        int budget = s.leafTestsPerStep;
        while (tHits) {
            const int k = __ffs(tHits) - 1;
            tHits &= tHits - 1u;
            if (tBase + static_cast<uint32_t>(k) >= static_cast<uint32_t>(s.triCount)) {
                if (errorFlags) atomicOr(errorFlags, 2u);
                continue;
            }
            const float4* tp = s.leafTris + 3 * (static_cast<size_t>(tBase) + static_cast<size_t>(k));
            const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, u, v;
            if (isectTri(r, a, b, c, tmin, AnyHit ? tmax : bt, t, u, v)) {
                if (AnyHit) { hit = true; return true; }
                const int idx = __float_as_int(a.w);
                if (best < 0 || t < bt || (t == bt && idx < best)) { best = idx; bt = t; bu = u; bv = v; }
            }
            if (--budget == 0) break;
        }
        if (tHits == 0u && (nBits >> 8) == 0u) {
            if (sp == 0) return true;
            const uint2 e = stack[--sp];
            if (e.y & kTriGroup) {   // a deferred leaf group: test it next, with no node work pending
                tBase = e.x;
                tHits = e.y & ~kTriGroup;
                nBits = 0;
            } else {
                nBase = e.x;
                nBits = e.y;
            }
        }
        return false;
    }
};

// ---------------------------------------------------------------- 8-wide traversal, 8 lanes per ray
// For the last bounces, whose few rays leave the GPU latency-bound, a group of
// eight lanes walks one ray: lane c decodes and tests child slot c of the
// fetched node (the same decode and slab test as WideWalk), tests the
// triangles of its slot when that slot is a leaf, and the group merges the
// candidates by (t, index).  The nearest internal child (lowest slot ^ octant
// key) is visited next; the others are pushed so that lower keys pop first.
// The stack is spread over the group: entry p lives in lane p % 8 at index
// p / 8 of that lane's own array, so a group holds 8 * kWideStack entries.
// Popped entries carry their entry distance and are dropped once it exceeds
// the current best by more than the box test's margins (the box would fail
// the test now).  Any order of visits gives the same result (closest hit is
// the minimum of (t, index) over all accepted triangles; culling is
// conservative), so this walk returns exactly what WideWalk returns.
// All eight lanes of a group must call it with the same ray.
template <bool AnyHit>
BTE_DI int traceWideGroup(const DevScene& s, const RayPre& r, float tmin, float tmax, uint2* stack,
                          unsigned int* errorFlags, float& tOut, float& uOut, float& vOut)
{
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int c = lane & 7;
    const unsigned gmask = 0xffu << (lane & ~7);
    const uint32_t oct = (r.ix < 0.0f ? 1u : 0u) | (r.iy < 0.0f ? 2u : 0u) | (r.iz < 0.0f ? 4u : 0u);
    int node = 0, sp = 0, visits = 0, best = -1;
    float bt = tmax, bu = 0.0f, bv = 0.0f;
    while (true) {
        if (node < 0) {
            if (sp == 0) break;
            --sp;
            const uint2 mine = stack[sp >> 3];
            const int e = __shfl_sync(gmask, static_cast<int>(mine.x), sp & 7, 8);
            const float te = __shfl_sync(gmask, __uint_as_float(mine.y), sp & 7, 8);
            if (!AnyHit && te > (bt * kCullMargin) * kBoxGrow) continue;
            node = e;
        }
        if (node >= s.wideNodeCount || ++visits > s.wideNodeCount) {   // never true for a built tree
            if (errorFlags && c == 0) atomicOr(errorFlags, 2u);
            break;
        }
        const float4* np = reinterpret_cast<const float4*>(s.wnodes) + 5 * static_cast<size_t>(node);
        const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2), f3 = __ldg(np + 3), f4 = __ldg(np + 4);
        const uint32_t em = __float_as_uint(f0.w);
        const uint32_t imask = em >> 24;
        // child slot c: the decode and slab test of WideWalk::step for one slot
        const float ax = wideScale(em & 0xffu) * r.ix, ay = wideScale((em >> 8) & 0xffu) * r.iy,
                    az = wideScale((em >> 16) & 0xffu) * r.iz;
        const float cx = (f0.x - r.ox) * r.ix, cy = (f0.y - r.oy) * r.iy, cz = (f0.z - r.oz) * r.iz;
        const float cnx = cx - r.px, cfx = cx + r.px, cny = cy - r.py, cfy = cy + r.py, cnz = cz - r.pz,
                    cfz = cz + r.pz;
        const bool sxn = oct & 1u, syn = oct & 2u, szn = oct & 4u;
        const bool hiWord = c >= 4;
        const uint32_t nx = __float_as_uint(sxn ? (hiWord ? f3.w : f3.z) : (hiWord ? f2.y : f2.x));
        const uint32_t fx = __float_as_uint(sxn ? (hiWord ? f2.y : f2.x) : (hiWord ? f3.w : f3.z));
        const uint32_t ny = __float_as_uint(syn ? (hiWord ? f4.y : f4.x) : (hiWord ? f2.w : f2.z));
        const uint32_t fy = __float_as_uint(syn ? (hiWord ? f2.w : f2.z) : (hiWord ? f4.y : f4.x));
        const uint32_t nz = __float_as_uint(szn ? (hiWord ? f4.w : f4.z) : (hiWord ? f3.y : f3.x));
        const uint32_t fz = __float_as_uint(szn ? (hiWord ? f3.y : f3.x) : (hiWord ? f4.w : f4.z));
        const float cull = AnyHit ? tmax * kCullMargin : bt * kCullMargin;
        const uint32_t sel = static_cast<uint32_t>(c & 3) | 0x7440u;
        const float tnx = __fmaf_rn(byteToFloat(nx, sel), ax, cnx);
        const float tfx = __fmaf_rn(byteToFloat(fx, sel), ax, cfx);
        const float tny = __fmaf_rn(byteToFloat(ny, sel), ay, cny);
        const float tfy = __fmaf_rn(byteToFloat(fy, sel), ay, cfy);
        const float tnz = __fmaf_rn(byteToFloat(nz, sel), az, cnz);
        const float tfz = __fmaf_rn(byteToFloat(fz, sel), az, cfz);
        const float tn = max3f(tnx, tny, fmaxf(tnz, tmin));
        const float tf = min3f(tfx, tfy, fminf(tfz, cull)) * kBoxGrow;
        const bool slotHit = tn <= tf;
        const bool internal = (imask >> c) & 1u;
        // the triangles of a leaf slot that was hit
        int lbest = -1;
        bool lhit = false;
        float lt = bt, lu = 0.0f, lv = 0.0f;
        if (slotHit && !internal) {
            const uint32_t mb = ((c >= 4 ? __float_as_uint(f1.w) : __float_as_uint(f1.z)) >> (8 * (c & 3))) & 0xffu;
            const int first = __float_as_int(f1.y) + static_cast<int>(mb & 31u);
            for (int k = 0; k < static_cast<int>(mb >> 5); ++k) {
                if (static_cast<uint32_t>(first + k) >= static_cast<uint32_t>(s.triCount)) {
                    if (errorFlags) atomicOr(errorFlags, 2u);
                    break;
                }
                const float4* tp = s.leafTris + 3 * static_cast<size_t>(first + k);
                const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
                float t, u, v;
                if (isectTri(r, a, b, cc, tmin, AnyHit ? tmax : lt, t, u, v)) {
                    if (AnyHit) { lhit = true; break; }
                    const int idx = __float_as_int(a.w);
                    if (lbest < 0 || t < lt || (t == lt && idx < lbest)) { lbest = idx; lt = t; lu = u; lv = v; }
                }
            }
        }
        if (AnyHit) {
            if (__any_sync(gmask, lhit)) { best = 1; break; }
        } else if (__any_sync(gmask, lbest >= 0)) {
            // group minimum of (t, index); lanes without a candidate hold (+inf, INT_MAX)
            float mt = lbest >= 0 ? lt : INFINITY;
            int mi = lbest >= 0 ? lbest : 0x7fffffff;
            float mu = lu, mv = lv;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const float ot = __shfl_xor_sync(gmask, mt, o, 8);
                const int oi = __shfl_xor_sync(gmask, mi, o, 8);
                const float ou = __shfl_xor_sync(gmask, mu, o, 8);
                const float ov = __shfl_xor_sync(gmask, mv, o, 8);
                if (ot < mt || (ot == mt && oi < mi)) { mt = ot; mi = oi; mu = ou; mv = ov; }
            }
            if (best < 0 || mt < bt || (mt == bt && mi < best)) { best = mi; bt = mt; bu = mu; bv = mv; }
        }
        // internal children hit, keyed slot ^ octant; the lowest key is visited next
        const uint32_t hits = (__ballot_sync(gmask, slotHit && internal) >> (lane & ~7)) & 0xffu;
        uint32_t keys = 0;
        for (uint32_t h = hits; h; h &= h - 1u) keys |= 1u << ((__ffs(h) - 1) ^ oct);
        if (keys == 0u) { node = -1; continue; }
        const uint32_t childBase = static_cast<uint32_t>(__float_as_int(f1.x));
        const uint32_t nearSlot = static_cast<uint32_t>(__ffs(keys) - 1) ^ oct;
        node = static_cast<int>(childBase) + __popc(imask & ((1u << nearSlot) - 1u));
        const uint32_t rest = keys & (keys - 1u);
        const int n = __popc(rest);
        if (n == 0) continue;
        if (sp + n > 8 * kWideStack) {
            if (errorFlags && c == 0) atomicOr(errorFlags, 1u);
            break;
        }
        // position sp + j (j = 0 .. n-1) holds the key of ascending rank n-1-j, so the lowest pops first;
        // this lane owns the position congruent to it mod 8
        const int j = (c - sp) & 7;
        uint32_t pick = rest;
        for (int q = 0; q < n - 1 - j && pick; ++q) pick &= pick - 1u;
        const uint32_t slot = (j < n && pick) ? (static_cast<uint32_t>(__ffs(pick) - 1) ^ oct) : static_cast<uint32_t>(c);
        const float tSlot = __shfl_sync(gmask, tn, static_cast<int>(slot), 8);
        if (j < n)
            stack[(sp + j) >> 3] = make_uint2(childBase + static_cast<uint32_t>(__popc(imask & ((1u << slot) - 1u))),
                                              __float_as_uint(tSlot));
        sp += n;
    }
    if (!AnyHit && best >= 0) { tOut = bt; uOut = bu; vOut = bv; }
    return best;
}

template <bool AnyHit>
BTE_DI int traceWide(const DevScene& s, const RayPre& r, float tmin, float tmax, float& tOut, float& uOut, float& vOut,
                     unsigned int* errorFlags)
{
    if (!r.valid || s.triCount <= 0) return -1;
    WideWalk<AnyHit> w;
    uint2 stack[kWideStack];
    w.start(r, tmin, tmax);
    while (!w.step(s, stack, errorFlags)) {
    }
    if (AnyHit) return w.hit ? 1 : -1;
    if (w.best >= 0) { tOut = w.bt; uOut = w.bu; vOut = w.bv; }
    return w.best;
}

// Dispatch on the tree the scene was built with (uniform across a launch).
template <int Width>
BTE_DI int traceClosestW(const DevScene& s, const RayPre& r, float tmin, float tmax, float& t, float& u, float& v,
                         unsigned int* errorFlags)
{
    if (Width == 8) return traceWide<false>(s, r, tmin, tmax, t, u, v, errorFlags);
    return traceClosest(s, r, tmin, tmax, t, u, v, errorFlags);
}
template <int Width>
BTE_DI bool traceOccludedW(const DevScene& s, const RayPre& r, float tmin, float tmax, unsigned int* errorFlags)
{
    if (Width == 8) {
        float t, u, v;
        return traceWide<true>(s, r, tmin, tmax, t, u, v, errorFlags) >= 0;
    }
    return traceOccluded(s, r, tmin, tmax, errorFlags);
}

}  // namespace bte
