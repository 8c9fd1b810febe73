// particle_common.cuh -- device helpers shared by the step kernels and the
// semi-implicit solver: stencil base and cell key of a particle, hardened Lame
// parameters, grid-node collision (box / sticky walls, level set).
#pragma once

#include "engine.cuh"
#include "mpm_math.cuh"

namespace mpm {

// Stencil base ceil(x/h - r) per axis (src/mpm_solver3d.cu:252-255).  Returns
// false when the stencil misses the grid in some axis (or x is not finite).
__device__ __forceinline__ bool stencilBase(const SceneDev& sc, const float* x, int* base) {
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float fb = ceilf(__fsub_rn(__fdiv_rn(x[a], sc.h), sc.range));
        bool ok = (fb >= (float)(1 - sc.S)) && (fb <= (float)(sc.res[a] - 1));
        inside = inside && ok;
        base[a] = ok ? (int)fb : 0;
    }
    return inside;
}

__device__ __forceinline__ uint32_t makeKey(const SceneDev& sc, const int* base) {
    int b[3], c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int t = base[a] + 4;
        b[a] = t >> 2;
        c[a] = t & 3;
    }
    uint32_t blk = sc.block_base + (uint32_t)((b[2] * sc.nb[1] + b[1]) * sc.nb[0] + b[0]);
    return (blk << 6) | (uint32_t)(c[2] << 4) | (uint32_t)(c[1] << 2) | (uint32_t)c[0];
}

// Lame parameters after hardening (src/material_point3d.cu:158-162).
__device__ __forceinline__ void plasticLame(const MaterialDev& m, const float* Fp, float& mu, float& la) {
    float Jp = det3(Fp);
    float f = expf(m.xi * (1.0f - Jp));
    mu = m.mu0 * f;
    la = m.lambda0 * f;
}

// Level-set collision object (LevelSetCollisionObject3D,
// include/collision_object3d.h:9-12, declared but not applied by the
// reference).  The signed distance is interpolated trilinearly at pos (clamped
// to the grid); where it is <= 0 the velocity relative to the collider's
// surface gets the friction law of applyBoundaryCollision
// (src/collision_object3d.cu:38-51) with the normalised trilinear gradient as
// the normal.
__device__ __forceinline__ float3 levelSetCollisionV(const SceneDev& sc, float px, float py, float pz, float vx, float vy,
                                                  float vz) {
    const float pos[3] = {px, py, pz};
    float vel[3] = {vx, vy, vz};
    int i0[3];
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float g = (pos[a] - sc.origin[a]) * sc.inv_h;
        g = fminf(fmaxf(g, 0.f), (float)(sc.res[a] - 1));
        i0[a] = min((int)g, sc.res[a] - 2);
        f[a] = g - (float)i0[a];
    }
    const size_t X = (size_t)sc.res[0], XY = X * (size_t)sc.res[1];
    const float* p0 = sc.phi + (size_t)i0[0] + X * (size_t)i0[1] + XY * (size_t)i0[2];
    float c[8];  // corner (dx, dy, dz) at index dx + 2 dy + 4 dz
#pragma unroll
    for (int k = 0; k < 8; ++k) c[k] = p0[(k & 1) + ((k >> 1) & 1) * X + ((k >> 2) & 1) * XY];
    float phi = 0.f, gr[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int d[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
        float w[3], s[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a] = d[a] ? f[a] : 1.f - f[a];
            s[a] = d[a] ? 1.f : -1.f;
        }
        phi += c[k] * (w[0] * w[1] * w[2]);
        gr[0] += c[k] * (s[0] * w[1] * w[2]);
        gr[1] += c[k] * (w[0] * s[1] * w[2]);
        gr[2] += c[k] * (w[0] * w[1] * s[2]);
    }
    if (phi > 0.f) return make_float3(vx, vy, vz);
    const float gn = sqrtf(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
    if (!(gn > 0.f)) return make_float3(vx, vy, vz);  // flat level set: no normal
    float n[3], rel[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        n[a] = gr[a] / gn;
        rel[a] = vel[a] - sc.phi_vel[a];
    }
    const float vn = rel[0] * n[0] + rel[1] * n[1] + rel[2] * n[2];
    if (vn >= kFltEps) return make_float3(vx, vy, vz);  // separating
    float vt[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) vt[a] = rel[a] - vn * n[a];
    const float vtn = sqrtf(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
    if (vtn <= -sc.phi_friction * vn + kFltEps) {
#pragma unroll
        for (int a = 0; a < 3; ++a) vel[a] = sc.phi_vel[a];
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) vel[a] = (vt[a] + sc.phi_friction * vn * (vt[a] / vtn)) + sc.phi_vel[a];
    }
    return make_float3(vel[0], vel[1], vel[2]);
}
__device__ __forceinline__ void levelSetCollision(const SceneDev& sc, const float* pos, float* vel) {
    const float3 r = levelSetCollisionV(sc, pos[0], pos[1], pos[2], vel[0], vel[1], vel[2]);
    vel[0] = r.x;
    vel[1] = r.y;
    vel[2] = r.z;
}

// The grid collision of one node (gridCollision, src/mpm_solver3d.cu:405-426,
// or the sticky-wall option), then the level set if the scene has one.
__device__ __forceinline__ void gridNodeCollision(const SceneDev& sc, const int* n, float dt, float* vs) {
    if (sc.boundary == MPM_BOUNDARY_STICKY) {
        bool wall = false;
#pragma unroll
        for (int a = 0; a < 3; ++a) wall |= (n[a] < sc.sticky) || (n[a] >= sc.res[a] - sc.sticky);
        if (wall) vs[0] = vs[1] = vs[2] = 0.f;
    } else {
        float pos[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) pos[a] = (sc.origin[a] + sc.h * (float)n[a]) + dt * vs[a];
        boundaryCollision(pos, vs, sc.origin, sc.target, sc.friction);
    }
    if (sc.phi) {
        float pos[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) pos[a] = (sc.origin[a] + sc.h * (float)n[a]) + dt * vs[a];
        levelSetCollision(sc, pos, vs);
    }
}

}  // namespace mpm
