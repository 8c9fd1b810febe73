// naive_mpm.cu -- reference-naive GPU restatement of the MPM snow step.
//
// A yardstick, not the product: it keeps the reference's execution model so
// that the B200 engine can be measured against it on the same GPU.
//   * AoS particles (128 B PIC-FLIP point, 236 B APIC point:
//     include/material_point3d.h:14-24, include/apic_material_point3d.h:14-24)
//     and AoS 52 B grid nodes (include/grid3d.h:28-32) over a dense res^3 grid;
//   * one thread per particle or per node, each sub-step its own launch
//     followed by a host synchronisation (thrust::for_each with
//     thrust::device, src/mpm_solver3d.cu:100-125);
//   * P2G scatters with seven float atomicAdd per (particle, node)
//     (src/mpm_solver3d.cu:237-294, src/apic_mpm_solver3d.cu:245-304) and
//     computes the particle's stress with its own SVD
//     (src/material_point3d.cu:33-45, 110-155);
//   * weights and gradients are evaluated per node with the reference's
//     double-literal 1D splines (src/interpolation3d.cu:88-142) over the
//     index range ceil(x/h - r) .. floor(x/h + r) with the in-grid test;
//   * G2P gathers whole 52 B nodes and updates Fe/Fp with a second SVD
//     (src/mpm_solver3d.cu:316-379, src/material_point3d.cu:53-70).
// Scene description and particle input are the library's own C structs, so
// both run the same workload.  Options the benchmark scenes use beyond the
// reference (gravity magnitude, sticky walls, prescribed V0) are honoured the
// same way as in the product.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <limits>
#include <vector>

#include "../../include/mpm_b200.h"
#include "../../mpm_b200/csrc/mpm_math.cuh"

namespace naive {

struct Point {              // MaterialPoint3D (128 B)
    float volume0, mass;
    float x[3], v[3];
    float Fe[9], Fp[9];     // row-major
    float mu0, lambda0, xi, theta_c, theta_s;
    int32_t model;
};
struct ApicPoint {          // APICMaterialPoint3D (236 B)
    Point p;
    float B[9], D[9], Dinv[9];
};
static_assert(sizeof(Point) == 128, "PIC-FLIP point is 128 B");
static_assert(sizeof(ApicPoint) == 236, "APIC point is 236 B");

struct Node {               // CollocatedGridData3D (52 B)
    int32_t index[3];
    float force[3];
    float velocity[3], velocity_star[3];
    float mass;
};
static_assert(sizeof(Node) == 52, "grid node is 52 B");

struct Settings {           // Grid3DSettings + Interpolator3D, read through device pointers
    float origin[3], target[3];
    int32_t res[3];
    float h, friction, range, gravity;
    int32_t interp, boundary, sticky;
};

constexpr float kEps = std::numeric_limits<float>::epsilon();

// 1D kernels with the reference's double literals (the float argument is
// promoted, the result rounded back to float).
__device__ float linN(float x) {
    float a = fabsf(x);
    return a < 1.0 ? 1.0 - a : 0.0;
}
__device__ float linNDot(float x) {
    float a = fabsf(x);
    return (a < 1.0 && a > kEps) ? -x / a : 0.0;
}
__device__ float quadN(float x) {
    float a = fabsf(x);
    if (a < 0.5) return 0.75 - a * a;
    if (a < 1.5) return 0.5 * pow(1.5 - a, 2);
    return 0.0;
}
__device__ float quadNDot(float x) {
    float a = fabsf(x);
    if (a < 0.5) return -2.0 * x;
    if (a < 1.5) return -(1.5 * x / a) + x;
    return 0.0;
}
__device__ float cubN(float x) {
    float a = fabsf(x);
    if (a < 1.0) return 0.5 * pow(a, 3) - a * a + 2.0 / 3.0;
    if (a < 2.0) return pow(2.0 - a, 3) / 6.0;
    return 0.0;
}
__device__ float cubNDot(float x) {
    float a = fabsf(x);
    if (a < 1.0) return 1.5 * x * a - 2.0 * x;
    if (a < 2.0) return -(2.0 * x / a) + 2.0 * x - 0.5 * (x * a);
    return 0.0;
}
__device__ float N1(int t, float x) { return t == MPM_INTERP_LINEAR ? linN(x) : t == MPM_INTERP_QUADRATIC_BSPLINE ? quadN(x) : cubN(x); }
__device__ float N1Dot(int t, float x) {
    return t == MPM_INTERP_LINEAR ? linNDot(x) : t == MPM_INTERP_QUADRATIC_BSPLINE ? quadNDot(x) : cubNDot(x);
}

// weight3D / weightGradient3D: distances recomputed per call, as in the reference.
__device__ float weight3D(const Settings* s, const float* xp, const float* xg) {
    float d[3];
    for (int a = 0; a < 3; ++a) d[a] = (xp[a] - xg[a]) / s->h;
    return N1(s->interp, d[0]) * N1(s->interp, d[1]) * N1(s->interp, d[2]);
}
__device__ void gradient3D(const Settings* s, const float* xp, const float* xg, float* g) {
    float d[3];
    for (int a = 0; a < 3; ++a) d[a] = (xp[a] - xg[a]) / s->h;
    const int t = s->interp;
    g[0] = (N1Dot(t, d[0]) * N1(t, d[1]) * N1(t, d[2])) / s->h;
    g[1] = (N1(t, d[0]) * N1Dot(t, d[1]) * N1(t, d[2])) / s->h;
    g[2] = (N1(t, d[0]) * N1(t, d[1]) * N1Dot(t, d[2])) / s->h;
}

__device__ void mul3(const float* A, const float* B, float* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
__device__ void mul3T(const float* A, const float* B, float* C) {  // A B^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
}

// -V0 * dPsi/dFe Fe^T (src/material_point3d.cu:33-45, 110-162).
__device__ void negVolumeStress(Point& p, float* P) {
    float Jp = mpm::det3(p.Fp);
    float f = exp(p.xi * (1.0 - Jp));
    float mu = p.mu0 * f, la = p.lambda0 * f;
    float U[9], s[3], V[9];
    mpm::svd3(p.Fe, U, s, V);
    if (p.model == MPM_MODEL_NEO_HOOKEAN) {
        float US[9], FeT[9];
        for (int i = 0; i < 3; ++i) s[i] = fmaxf(s[i], kEps);
        for (int i = 0; i < 9; ++i) US[i] = U[i] * s[i % 3];
        mul3T(US, V, p.Fe);
        float Je = mpm::det3(p.Fe);
        mul3T(p.Fe, p.Fe, FeT);
        float l = la * log(Je);
        for (int i = 0; i < 9; ++i) P[i] = mu * FeT[i];
        for (int i = 0; i < 3; ++i) P[4 * i] += l - mu;
    } else {
        float R[9], D[9];
        mul3T(U, V, R);
        float Je = mpm::det3(p.Fe);
        for (int i = 0; i < 9; ++i) D[i] = p.Fe[i] - R[i];
        mul3T(D, p.Fe, P);
        float two_mu = 2.0 * mu, lj = la * (Je - 1.0) * Je;
        for (int i = 0; i < 9; ++i) P[i] *= two_mu;
        for (int i = 0; i < 3; ++i) P[4 * i] += lj;
    }
    for (int i = 0; i < 9; ++i) P[i] = -(p.volume0 * P[i]);
}

// updateDeformationGradient (src/material_point3d.cu:53-70).
__device__ void updateDeformation(Point& p, const float* gradv, float dt) {
    float A[9], Fe[9], F[9];
    for (int i = 0; i < 9; ++i) A[i] = (i % 4 == 0 ? 1.0f : 0.0f) + dt * gradv[i];
    mul3(A, p.Fe, Fe);
    mul3(Fe, p.Fp, F);
    float U[9], s[3], V[9];
    mpm::svd3(Fe, U, s, V);
    for (int i = 0; i < 3; ++i) s[i] = fmaxf(fminf(s[i], 1.0f + p.theta_s), 1.0f - p.theta_c);
    float US[9], VSi[9], T[9];
    for (int i = 0; i < 9; ++i) {
        US[i] = U[i] * s[i % 3];
        VSi[i] = V[i] / s[i % 3];
    }
    mul3T(US, V, p.Fe);
    mul3T(VSi, U, T);
    mul3(T, F, p.Fp);
}

template <class P>
__device__ Point& base(P& q);
template <>
__device__ Point& base<Point>(Point& q) { return q; }
template <>
__device__ Point& base<ApicPoint>(ApicPoint& q) { return q.p; }

#define NODE_LOOP(s, xp, ...)                                                                            \
    {                                                                                                    \
        int lo_[3], hi_[3];                                                                              \
        for (int a_ = 0; a_ < 3; ++a_) {                                                                 \
            lo_[a_] = (int)ceilf(xp[a_] / s->h - s->range);                                              \
            hi_[a_] = (int)floorf(xp[a_] / s->h + s->range);                                             \
            /* out-of-grid nodes are skipped below anyway; clamping keeps */                             \
            /* the loop finite for non-finite positions */                                               \
            lo_[a_] = max(lo_[a_], 0);                                                                   \
            hi_[a_] = min(hi_[a_], s->res[a_] - 1);                                                      \
        }                                                                                                \
        for (int gx = lo_[0]; gx <= hi_[0]; ++gx)                                                        \
            for (int gy = lo_[1]; gy <= hi_[1]; ++gy)                                                    \
                for (int gz = lo_[2]; gz <= hi_[2]; ++gz) {                                              \
                    if (gx < 0 || gx >= s->res[0] || gy < 0 || gy >= s->res[1] || gz < 0 || gz >= s->res[2]) \
                        continue;                                                                        \
                    const size_t gi = (size_t)gx + (size_t)s->res[0] * ((size_t)gy + (size_t)s->res[1] * gz); \
                    const float gp[3] = {s->origin[0] + s->h * (float)gx, s->origin[1] + s->h * (float)gy,  \
                                         s->origin[2] + s->h * (float)gz};                               \
                    __VA_ARGS__                                                                          \
                }                                                                                        \
    }

template <class P>
__global__ void p2gMassKernel(P* pts, size_t n, Node* grid, const Settings* s) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Point& p = base(pts[i]);
    NODE_LOOP(s, p.x, { atomicAdd(&grid[gi].mass, p.mass * weight3D(s, p.x, gp)); })
}

template <class P>
__global__ void g2pVolumeKernel(P* pts, size_t n, const Node* grid, const Settings* s) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Point& p = base(pts[i]);
    float dens = 0.0f;
    const float inv = 1.0 / (s->h * s->h * s->h);
    NODE_LOOP(s, p.x, { dens += grid[gi].mass * weight3D(s, p.x, gp) * inv; })
    p.volume0 = p.mass / dens;
}

__global__ void resetKernel(Node* grid, size_t nn) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    Node& g = grid[i];
    g.mass = 0.0f;
    for (int a = 0; a < 3; ++a) g.force[a] = g.velocity[a] = g.velocity_star[a] = 0.0f;
}

template <bool APIC, class P>
__global__ void p2gKernel(P* pts, size_t n, Node* grid, const Settings* s) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    P& q = pts[i];
    Point& p = base(q);
    float C[9];
    if constexpr (APIC) mul3(q.B, q.Dinv, C);
    float sig[9];
    negVolumeStress(p, sig);
    NODE_LOOP(s, p.x, {
        const float w = weight3D(s, p.x, gp);
        float g[3];
        gradient3D(s, p.x, gp, g);
        const float m = p.mass * w;
        float vi[3];
        if constexpr (APIC) {
            float r[3] = {gp[0] - p.x[0], gp[1] - p.x[1], gp[2] - p.x[2]};
            for (int a = 0; a < 3; ++a) vi[a] = m * (p.v[a] + (C[3 * a] * r[0] + C[3 * a + 1] * r[1] + C[3 * a + 2] * r[2]));
        } else {
            for (int a = 0; a < 3; ++a) vi[a] = p.v[a] * m;
        }
        Node& nd = grid[gi];
        atomicAdd(&nd.mass, m);
        for (int a = 0; a < 3; ++a) atomicAdd(&nd.velocity[a], vi[a]);
        for (int a = 0; a < 3; ++a) atomicAdd(&nd.force[a], sig[3 * a] * g[0] + sig[3 * a + 1] * g[1] + sig[3 * a + 2] * g[2]);
    })
}

__global__ void gravityKernel(Node* grid, size_t nn, const Settings* s) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    Node& g = grid[i];
    if (g.mass > kEps) g.force[1] -= s->gravity * g.mass;
}

__global__ void updateKernel(Node* grid, size_t nn, float dt) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    Node& g = grid[i];
    if (g.mass > kEps) {
        for (int a = 0; a < 3; ++a) g.velocity[a] /= g.mass;
        for (int a = 0; a < 3; ++a) g.velocity_star[a] = g.velocity[a] + dt * g.force[a] / g.mass;
    }
}

__global__ void gridCollisionKernel(Node* grid, size_t nn, const Settings* s, float dt) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    Node& g = grid[i];
    if (s->boundary == MPM_BOUNDARY_STICKY) {
        bool wall = false;
        for (int a = 0; a < 3; ++a) wall |= (g.index[a] < s->sticky) || (g.index[a] >= s->res[a] - s->sticky);
        if (wall) g.velocity_star[0] = g.velocity_star[1] = g.velocity_star[2] = 0.0f;
        return;
    }
    float pos[3];
    for (int a = 0; a < 3; ++a) pos[a] = (s->origin[a] + s->h * (float)g.index[a]) + dt * g.velocity_star[a];
    mpm::boundaryCollision(pos, g.velocity_star, s->origin, s->target, s->friction);
}

template <bool APIC, class P>
__global__ void g2pKernel(P* pts, size_t n, const Node* grid, const Settings* s, float dt, float blend) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    P& q = pts[i];
    Point& p = base(q);
    float gradv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, vpic[3] = {0, 0, 0}, vflip[3] = {p.v[0], p.v[1], p.v[2]};
    float B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    NODE_LOOP(s, p.x, {
        const float w = weight3D(s, p.x, gp);
        float g[3];
        gradient3D(s, p.x, gp, g);
        const Node nd = grid[gi];
        float vi[3];
        for (int a = 0; a < 3; ++a) vi[a] = nd.velocity_star[a] * w;
        for (int a = 0; a < 3; ++a) vpic[a] += vi[a];
        if constexpr (APIC) {
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) B[3 * a + b] += vi[a] * (gp[b] - p.x[b]);
        } else {
            for (int a = 0; a < 3; ++a) vflip[a] += (nd.velocity_star[a] - nd.velocity[a]) * w;
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) gradv[3 * a + b] += nd.velocity_star[a] * g[b];
    })
    float vel[3];
    if constexpr (APIC) {
        for (int a = 0; a < 9; ++a) q.B[a] = B[a];
        for (int a = 0; a < 3; ++a) vel[a] = vpic[a];
    } else {
        const float om = 1.0 - blend;
        for (int a = 0; a < 3; ++a) vel[a] = blend * vflip[a] + om * vpic[a];
    }
    updateDeformation(p, gradv, dt);
    for (int a = 0; a < 3; ++a) p.v[a] = vel[a];
}

template <class P>
__global__ void particlesCollisionKernel(P* pts, size_t n, const Settings* s, float dt) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Point& p = base(pts[i]);
    float pos[3];
    for (int a = 0; a < 3; ++a) pos[a] = p.x[a] + dt * p.v[a];
    mpm::boundaryCollision(pos, p.v, s->origin, s->target, s->friction);
}

template <class P>
__global__ void advectKernel(P* pts, size_t n, float dt) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Point& p = base(pts[i]);
    for (int a = 0; a < 3; ++a) p.x[a] += dt * p.v[a];
}

__global__ void gatherKernel(const char* pts, size_t stride, size_t n, int offset_words, int comps, float* out) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* src = reinterpret_cast<const float*>(pts + i * stride) + offset_words;
    for (int c = 0; c < comps; ++c) out[i * comps + c] = src[c];
}

struct Solver {
    mpm_scene_desc desc{};
    size_t n = 0, nn = 0;
    bool apic = false;
    void* pts = nullptr;
    Node* grid = nullptr;
    Settings* settings = nullptr;
    float* scratch = nullptr;
    cudaEvent_t ev[2]{};
};

static thread_local char g_err[512];

static int fail(const char* what, cudaError_t e) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return (int)MPM_ERR_CUDA;
}

#define NV_TRY(what, call)                          \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return naive::fail(what, e_); \
    } while (0)

// Every sub-step is one launch followed by a synchronisation, as thrust::for_each
// with the thrust::device policy does.
#define NV_LAUNCH(what, ...)                          \
    do {                                              \
        __VA_ARGS__;                                  \
        NV_TRY(what, cudaGetLastError());             \
        NV_TRY(what, cudaStreamSynchronize(0));       \
    } while (0)

static unsigned blocksFor(size_t n) { return (unsigned)((n + 255) / 256); }

template <bool APIC, class P>
static int stepT(Solver& s) {
    const float dt = s.desc.dt;
    P* pts = static_cast<P*>(s.pts);
    NV_LAUNCH("resetGrid", resetKernel<<<blocksFor(s.nn), 256>>>(s.grid, s.nn));
    NV_LAUNCH("particlesToGrid", (p2gKernel<APIC, P><<<blocksFor(s.n), 256>>>(pts, s.n, s.grid, s.settings)));
    NV_LAUNCH("computeGravityForces", gravityKernel<<<blocksFor(s.nn), 256>>>(s.grid, s.nn, s.settings));
    NV_LAUNCH("updateGridVelocities", updateKernel<<<blocksFor(s.nn), 256>>>(s.grid, s.nn, dt));
    NV_LAUNCH("gridCollision", gridCollisionKernel<<<blocksFor(s.nn), 256>>>(s.grid, s.nn, s.settings, dt));
    NV_LAUNCH("gridToParticles",
              (g2pKernel<APIC, P><<<blocksFor(s.n), 256>>>(pts, s.n, s.grid, s.settings, dt, s.desc.blend)));
    if (s.desc.particles_collision)
        NV_LAUNCH("particlesCollision", particlesCollisionKernel<P><<<blocksFor(s.n), 256>>>(pts, s.n, s.settings, dt));
    NV_LAUNCH("advectParticles", advectKernel<P><<<blocksFor(s.n), 256>>>(pts, s.n, dt));
    return 0;
}

template <class P>
static int initializeT(Solver& s) {
    P* pts = static_cast<P*>(s.pts);
    NV_LAUNCH("resetGrid", resetKernel<<<blocksFor(s.nn), 256>>>(s.grid, s.nn));
    NV_LAUNCH("P2GMass", p2gMassKernel<P><<<blocksFor(s.n), 256>>>(pts, s.n, s.grid, s.settings));
    if (s.desc.volume_mode != MPM_VOLUME_PRESCRIBED)
        NV_LAUNCH("G2PVolume", g2pVolumeKernel<P><<<blocksFor(s.n), 256>>>(pts, s.n, s.grid, s.settings));
    return 0;
}

static void fillPoint(Point& p, const mpm_particles_in* in, size_t i, const mpm_scene_desc* d) {
    const int mi = in->material ? in->material[i] : 0;
    const mpm_material& m = in->materials[mi];
    for (int a = 0; a < 3; ++a) {
        p.x[a] = in->position[3 * i + a];
        p.v[a] = in->velocity[3 * i + a];
    }
    p.mass = in->mass[i];
    p.volume0 = (d->volume_mode == MPM_VOLUME_PRESCRIBED && in->volume) ? in->volume[i] : 0.0f;
    for (int k = 0; k < 9; ++k) p.Fe[k] = p.Fp[k] = (k % 4 == 0) ? 1.0f : 0.0f;
    // src/material_point3d.cu:25-26
    p.mu0 = m.youngs_modulus / (2.0 * (1.0 + m.poisson_ratio));
    p.lambda0 = (m.youngs_modulus * m.poisson_ratio) / ((1.0 + m.poisson_ratio) * (1.0 - 2.0 * m.poisson_ratio));
    p.xi = m.hardening;
    p.theta_c = m.critical_compression;
    p.theta_s = m.critical_stretch;
    p.model = m.model;
}

}  // namespace naive

using naive::Solver;

extern "C" {

MPM_API const char* naive_last_error(void) { return naive::g_err; }

MPM_API int naive_create(const mpm_scene_desc* d, const mpm_particles_in* in, void** out) {
    using namespace naive;
    if (!d || !in || !out || (in->n && (!in->position || !in->velocity || !in->mass || !in->materials))) {
        snprintf(g_err, sizeof g_err, "invalid argument");
        return (int)MPM_ERR_INVALID_ARG;
    }
    if (d->transfer == MPM_TRANSFER_APIC && d->interpolation == MPM_INTERP_LINEAR) {
        snprintf(g_err, sizeof g_err, "APIC with linear interpolation is singular");
        return (int)MPM_ERR_INVALID_ARG;
    }
    Solver* s = new Solver();
    s->desc = *d;
    s->n = in->n;
    s->nn = (size_t)d->resolution[0] * d->resolution[1] * d->resolution[2];
    s->apic = d->transfer == MPM_TRANSFER_APIC;
    Settings st{};
    for (int a = 0; a < 3; ++a) {
        st.origin[a] = d->origin[a];
        st.res[a] = d->resolution[a];
        st.target[a] = d->origin[a] + d->stride * (float)d->resolution[a];
    }
    st.h = d->stride;
    st.friction = d->friction;
    st.range = d->interpolation == MPM_INTERP_LINEAR ? 1.0f : d->interpolation == MPM_INTERP_QUADRATIC_BSPLINE ? 1.5f : 2.0f;
    st.gravity = d->gravity;
    st.interp = d->interpolation;
    st.boundary = d->boundary;
    st.sticky = d->sticky_cells;
    const size_t psize = s->apic ? sizeof(ApicPoint) : sizeof(Point);
    std::vector<char> host(psize * (s->n ? s->n : 1));
    float k = 0.0f;
    if (d->interpolation == MPM_INTERP_CUBIC_BSPLINE) k = 1 / 3.0;
    if (d->interpolation == MPM_INTERP_QUADRATIC_BSPLINE) k = 1 / 4.0;
    const float D = k * d->stride * d->stride;
    for (size_t i = 0; i < s->n; ++i) {
        if (s->apic) {
            ApicPoint& q = reinterpret_cast<ApicPoint*>(host.data())[i];
            fillPoint(q.p, in, i, d);
            for (int j = 0; j < 9; ++j) {
                q.B[j] = 0.0f;
                q.D[j] = (j % 4 == 0) ? D : 0.0f;
                q.Dinv[j] = (j % 4 == 0) ? 1.0f / D : 0.0f;
            }
        } else {
            fillPoint(reinterpret_cast<Point*>(host.data())[i], in, i, d);
        }
    }
    std::vector<Node> g(s->nn);
    for (int z = 0; z < d->resolution[2]; ++z)
        for (int y = 0; y < d->resolution[1]; ++y)
            for (int x = 0; x < d->resolution[0]; ++x) {
                Node& nd = g[(size_t)x + (size_t)d->resolution[0] * ((size_t)y + (size_t)d->resolution[1] * z)];
                nd = Node{};
                nd.index[0] = x;
                nd.index[1] = y;
                nd.index[2] = z;
            }
    int rc = 0;
    auto chk = [&](const char* what, cudaError_t e) {
        if (e != cudaSuccess && rc == 0) rc = fail(what, e);
    };
    chk("cudaMalloc", cudaMalloc(&s->pts, host.size()));
    chk("cudaMalloc", cudaMalloc(&s->grid, sizeof(Node) * s->nn));
    chk("cudaMalloc", cudaMalloc(&s->settings, sizeof(Settings)));
    chk("cudaMalloc", cudaMalloc(&s->scratch, sizeof(float) * 9 * (s->n ? s->n : 1)));
    if (!rc) chk("cudaMemcpy", cudaMemcpy(s->pts, host.data(), host.size(), cudaMemcpyHostToDevice));
    if (!rc) chk("cudaMemcpy", cudaMemcpy(s->grid, g.data(), sizeof(Node) * s->nn, cudaMemcpyHostToDevice));
    if (!rc) chk("cudaMemcpy", cudaMemcpy(s->settings, &st, sizeof st, cudaMemcpyHostToDevice));
    if (!rc) chk("cudaEventCreate", cudaEventCreate(&s->ev[0]));
    if (!rc) chk("cudaEventCreate", cudaEventCreate(&s->ev[1]));
    if (!rc && s->n) rc = s->apic ? initializeT<ApicPoint>(*s) : initializeT<Point>(*s);
    if (rc) {
        cudaFree(s->pts);
        cudaFree(s->grid);
        cudaFree(s->settings);
        cudaFree(s->scratch);
        delete s;
        return rc;
    }
    *out = s;
    return 0;
}

MPM_API int naive_destroy(void* h) {
    Solver* s = static_cast<Solver*>(h);
    if (!s) return 0;
    cudaFree(s->pts);
    cudaFree(s->grid);
    cudaFree(s->settings);
    cudaFree(s->scratch);
    if (s->ev[0]) cudaEventDestroy(s->ev[0]);
    if (s->ev[1]) cudaEventDestroy(s->ev[1]);
    delete s;
    return 0;
}

MPM_API int naive_step(void* h, int32_t nsteps) {
    Solver* s = static_cast<Solver*>(h);
    if (!s || nsteps < 0) return (int)MPM_ERR_INVALID_ARG;
    if (!s->n) return 0;
    for (int k = 0; k < nsteps; ++k) {
        int rc = s->apic ? naive::stepT<true, naive::ApicPoint>(*s) : naive::stepT<false, naive::Point>(*s);
        if (rc) return rc;
    }
    return 0;
}

// nsteps steps between two events on the legacy stream; *ms = their distance.
MPM_API int naive_timed_step(void* h, int32_t nsteps, float* ms) {
    Solver* s = static_cast<Solver*>(h);
    if (!s || !ms) return (int)MPM_ERR_INVALID_ARG;
    NV_TRY("cudaEventRecord", cudaEventRecord(s->ev[0], 0));
    int rc = naive_step(h, nsteps);
    if (rc) return rc;
    NV_TRY("cudaEventRecord", cudaEventRecord(s->ev[1], 0));
    NV_TRY("cudaEventSynchronize", cudaEventSynchronize(s->ev[1]));
    NV_TRY("cudaEventElapsedTime", cudaEventElapsedTime(ms, s->ev[0], s->ev[1]));
    return 0;
}

// field: MPM_FIELD_POSITION, VELOCITY, FE, FP, B (APIC), VOLUME0, MASS, in input order.
MPM_API int naive_download(void* h, int32_t field, float* host) {
    Solver* s = static_cast<Solver*>(h);
    if (!s || !host) return (int)MPM_ERR_INVALID_ARG;
    int off = -1, comps = 0;
    switch (field) {
    case MPM_FIELD_POSITION: off = offsetof(naive::Point, x) / 4, comps = 3; break;
    case MPM_FIELD_VELOCITY: off = offsetof(naive::Point, v) / 4, comps = 3; break;
    case MPM_FIELD_FE: off = offsetof(naive::Point, Fe) / 4, comps = 9; break;
    case MPM_FIELD_FP: off = offsetof(naive::Point, Fp) / 4, comps = 9; break;
    case MPM_FIELD_VOLUME0: off = offsetof(naive::Point, volume0) / 4, comps = 1; break;
    case MPM_FIELD_MASS: off = offsetof(naive::Point, mass) / 4, comps = 1; break;
    case MPM_FIELD_B:
        if (s->apic) off = offsetof(naive::ApicPoint, B) / 4, comps = 9;
        break;
    default: break;
    }
    if (off < 0) {
        snprintf(naive::g_err, sizeof naive::g_err, "unsupported field %d", field);
        return (int)MPM_ERR_INVALID_ARG;
    }
    if (!s->n) return 0;
    const size_t stride = s->apic ? sizeof(naive::ApicPoint) : sizeof(naive::Point);
    NV_LAUNCH("gather", naive::gatherKernel<<<naive::blocksFor(s->n), 256>>>(static_cast<const char*>(s->pts), stride,
                                                                           s->n, off, comps, s->scratch));
    NV_TRY("cudaMemcpy", cudaMemcpy(host, s->scratch, sizeof(float) * comps * s->n, cudaMemcpyDeviceToHost));
    return 0;
}

}  // extern "C"
