// bte_trace.cuh -- ray traversal: watertight ray/triangle test and BVH2 walk.
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

constexpr int kTraversalStack = 96;

struct RayPre {
    float ox, oy, oz;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    float ix, iy, iz;     // reciprocal direction for the slab test (zeros replaced by +-1e-30)
    float px, py, pz;     // per-slab widening in t units
    float nx, ny, nz;     // -origin * reciprocal direction (slab test in fused form)
    bool valid;
};

constexpr float kTriErrK = 64.0f;

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

// Watertight test; returns true with t in [tmin, tmax].
BTE_DI bool isectTri(const RayPre& r, float4 a, float4 b, float4 c, float tmin, float tmax, float& ot, float& ou,
                     float& ov)
{
    const float Ax0 = a.x - r.ox, Ay0 = a.y - r.oy, Az0 = a.z - r.oz;
    const float Bx0 = b.x - r.ox, By0 = b.y - r.oy, Bz0 = b.z - r.oz;
    const float Cx0 = c.x - r.ox, Cy0 = c.y - r.oy, Cz0 = c.z - r.oz;
    const float Akz = comp3(Ax0, Ay0, Az0, r.kz), Bkz = comp3(Bx0, By0, Bz0, r.kz), Ckz = comp3(Cx0, Cy0, Cz0, r.kz);
    const float Ax = comp3(Ax0, Ay0, Az0, r.kx) - r.Sx * Akz;
    const float Ay = comp3(Ax0, Ay0, Az0, r.ky) - r.Sy * Akz;
    const float Bx = comp3(Bx0, By0, Bz0, r.kx) - r.Sx * Bkz;
    const float By = comp3(Bx0, By0, Bz0, r.ky) - r.Sy * Bkz;
    const float Cx = comp3(Cx0, Cy0, Cz0, r.kx) - r.Sx * Ckz;
    const float Cy = comp3(Cx0, Cy0, Cz0, r.ky) - r.Sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = static_cast<float>(static_cast<double>(Cx) * static_cast<double>(By) - static_cast<double>(Cy) * static_cast<double>(Bx));
        V = static_cast<float>(static_cast<double>(Ax) * static_cast<double>(Cy) - static_cast<double>(Ay) * static_cast<double>(Cx));
        W = static_cast<float>(static_cast<double>(Bx) * static_cast<double>(Ay) - static_cast<double>(By) * static_cast<double>(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = r.Sz * Akz, Bz = r.Sz * Bkz, Cz = r.Sz * Ckz;
    const float T = U * Az + V * Bz + W * Cz;
    const float t = T / det;
    if (!(t >= tmin && t <= tmax)) return false;
    ot = t;
    ou = V / det;
    ov = W / det;
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

}  // namespace bte
