// mpm_math.cuh -- per-particle math of the snow step, FP32, register resident.
//
// Splines follow Interpolator3D (src/interpolation3d.cu:88-142), the 3x3 SVD
// follows the method of the reference's 3x3_SVD_CUDA dependency (McAdams,
// Selle, Tamstorf, Teran, Sifakis, UW-Madison CS TR-1690, 2011), boundary
// collision follows applyBoundaryCollision (src/collision_object3d.cu:7-54).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace mpm {

constexpr float kFltEps = 1.1920928955078125e-07f;  // std::numeric_limits<float>::epsilon()
constexpr int kSvdSweeps = 5;

// ---------------------------------------------------------------------------
// 1D B-spline kernels.  d is the signed distance in cells.  Where the
// reference's double-literal expression can be reproduced exactly in FP32
// (linear, quadratic) it is; the cubic forms are within ~2 ulp of it.
// ---------------------------------------------------------------------------
template <int S>
__device__ __forceinline__ float splineN(float d);
template <int S>
__device__ __forceinline__ float splineNDot(float d);

template <>
__device__ __forceinline__ float splineN<2>(float d) {
    float t = fabsf(d);
    return t < 1.0f ? 1.0f - t : 0.0f;
}
template <>
__device__ __forceinline__ float splineNDot<2>(float d) {
    float t = fabsf(d);
    return (t < 1.0f && t > kFltEps) ? -d / t : 0.0f;
}
template <>
__device__ __forceinline__ float splineN<3>(float d) {
    float t = fabsf(d);
    if (t < 0.5f) return __fsub_rn(0.75f, __fmul_rn(t, t));
    if (t < 1.5f) {
        float u = 1.5f - t;  // exact
        return __fmul_rn(0.5f, __fmul_rn(u, u));
    }
    return 0.0f;
}
template <>
__device__ __forceinline__ float splineNDot<3>(float d) {
    float t = fabsf(d);
    if (t < 0.5f) return -2.0f * d;
    if (t < 1.5f) return __fsub_rn(d, copysignf(1.5f, d));
    return 0.0f;
}
template <>
__device__ __forceinline__ float splineN<4>(float d) {
    float t = fabsf(d);
    if (t < 1.0f) return fmaf(fmaf(0.5f, t, -1.0f) * t, t, 0.66666666666666667f);
    if (t < 2.0f) {
        float u = 2.0f - t;
        return u * u * u * 0.16666666666666667f;
    }
    return 0.0f;
}
template <>
__device__ __forceinline__ float splineNDot<4>(float d) {
    float t = fabsf(d);
    if (t < 1.0f) return d * fmaf(1.5f, t, -2.0f);
    if (t < 2.0f) {
        float u = 2.0f - t;
        return -copysignf(0.5f * u * u, d);  // -sign(d) (2-|d|)^2 / 2
    }
    return 0.0f;
}

template <int S>
__device__ __forceinline__ float splineRange() {
    return S == 2 ? 1.0f : (S == 3 ? 1.5f : 2.0f);
}

// All S weights (and derivatives, in cells) of one axis for a stencil that
// starts at base = ceil(x/h - r), so that d0 = x/h - base lies in (r-1, r].
// Node k sits at distance d0 - k, whose sign and spline piece are known in
// advance, so the piecewise kernels need no branches.  The values are those of
// splineN / splineNDot (the pieces agree at their junctions); the linear
// kernel keeps the branchy form for the reference's zero derivative at
// |d| = 0 and |d| = 1.
// d[k] is the distance (in cells) of stencil node k; pass d[k] = d[0] - k
// when the per-node rounding of (x - o - h i)/h is not needed.
template <int S>
__device__ __forceinline__ void splineWeights(const float* d, float* w, float* dw);

template <>
__device__ __forceinline__ void splineWeights<2>(const float* d, float* w, float* dw) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        w[k] = splineN<2>(d[k]);
        dw[k] = splineNDot<2>(d[k]);
    }
}

template <>
__device__ __forceinline__ void splineWeights<3>(const float* d, float* w, float* dw) {
    // d0 in (0.5, 1.5] (outer piece), d1 in (-0.5, 0.5] (inner), d2 in (-1.5, -0.5] (outer)
    const float u0 = 1.5f - d[0];        // >= 0
    const float d1 = d[1];
    const float u2 = 1.5f + d[2];        // 1.5 - |d2|, >= 0
    w[0] = 0.5f * u0 * u0;
    w[1] = 0.75f - d1 * d1;
    w[2] = 0.5f * u2 * u2;
    dw[0] = -u0;                          // d - 1.5 sign(d), d > 0
    dw[1] = -2.0f * d1;
    dw[2] = u2;                           // d + 1.5, d < 0
}

template <>
__device__ __forceinline__ void splineWeights<4>(const float* d, float* w, float* dw) {
    // d0 in (1, 2] (outer), d1 in (0, 1] (inner), d2 in (-1, 0] (inner), d3 in (-2, -1] (outer)
    const float u0 = 2.0f - d[0];        // >= 0
    const float t1 = d[1];               // |d1|
    const float t2 = -d[2];              // |d2|
    const float u3 = 2.0f + d[3];        // 2 - |d3|
    const float sixth = 0.16666666666666667f, twothirds = 0.66666666666666667f;
    w[0] = u0 * u0 * u0 * sixth;
    w[1] = fmaf(fmaf(0.5f, t1, -1.0f) * t1, t1, twothirds);
    w[2] = fmaf(fmaf(0.5f, t2, -1.0f) * t2, t2, twothirds);
    w[3] = u3 * u3 * u3 * sixth;
    dw[0] = -0.5f * u0 * u0;             // d > 0 outer: -(2-|d|)^2 / 2
    dw[1] = t1 * fmaf(1.5f, t1, -2.0f);  // d > 0 inner: d (1.5|d| - 2)
    dw[2] = -t2 * fmaf(1.5f, t2, -2.0f); // d <= 0 inner
    dw[3] = 0.5f * u3 * u3;              // d < 0 outer: +(2-|d|)^2 / 2
}

// ---------------------------------------------------------------------------
// Small row-major 3x3 helpers.
// ---------------------------------------------------------------------------
struct M3 {
    float a[9];
};

__device__ __forceinline__ float det3(const float* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

__device__ __forceinline__ void matmul3(const float* A, const float* B, float* C) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = fmaf(A[3 * i + 2], B[6 + j], fmaf(A[3 * i + 1], B[3 + j], A[3 * i] * B[j]));
}

// ---------------------------------------------------------------------------
// 3x3 SVD, McAdams et al. 2011: Jacobi eigen-analysis of A^T A with
// approximate Givens rotations, sort of the columns of A V with sign fixes,
// Givens QR.  The reference's library runs 4 Jacobi sweeps; for nearly equal
// singular values (Fe close to a rotation, the common case in snow) 4 sweeps
// can leave off-diagonal residues up to ~1e-5, so 5 are run here (the FP32
// floor of the method, ~5e-7 reconstruction error, is reached by then).  A = U diag(s) V^T, U and V rotations, s sorted by
// decreasing magnitude, s[2] carrying the sign of det(A).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void jacobiRotate(float (&S)[3][3], float* V, int p, int q) {
    const float gamma = 5.82842712474619f;  // 3 + 2 sqrt(2)
    const float cstar = 0.923879532511287f;  // cos(pi/8)
    const float sstar = 0.382683432365090f;  // sin(pi/8)
    float ch = 2.0f * (S[p][p] - S[q][q]);
    float sh = S[p][q];
    bool b = gamma * sh * sh < ch * ch;
    float w = rsqrtf(fmaf(ch, ch, sh * sh));
    ch = b ? w * ch : cstar;
    sh = b ? w * sh : sstar;
    float c = fmaf(ch, ch, -sh * sh);
    float s = 2.0f * ch * sh;
    // S <- G^T S G with G the (p, q) rotation; S is symmetric, so only its
    // upper triangle is formed (r is the third index; S[r][r] is unchanged).
    const int r = 3 - p - q;
    const float spp = S[p][p], sqq = S[q][q], spq = S[p][q], spr = S[p][r], sqr = S[q][r];
    const float cc = c * c, ss = s * s, cs = c * s;
    const float t = 2.0f * cs * spq;
    S[p][p] = fmaf(cc, spp, fmaf(ss, sqq, t));
    S[q][q] = fmaf(ss, spp, fmaf(cc, sqq, -t));
    S[p][q] = S[q][p] = fmaf(cc - ss, spq, cs * (sqq - spp));
    S[p][r] = S[r][p] = fmaf(c, spr, s * sqr);
    S[q][r] = S[r][q] = fmaf(-s, spr, c * sqr);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float vp = V[3 * k + p], vq = V[3 * k + q];
        V[3 * k + p] = fmaf(c, vp, s * vq);
        V[3 * k + q] = fmaf(-s, vp, c * vq);
    }
}

__device__ __forceinline__ void condSwapNeg(bool cond, float* B, float* V, int i, int j) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float bi = B[3 * k + i], bj = B[3 * k + j];
        B[3 * k + i] = cond ? bj : bi;
        B[3 * k + j] = cond ? -bi : bj;
        float vi = V[3 * k + i], vj = V[3 * k + j];
        V[3 * k + i] = cond ? vj : vi;
        V[3 * k + j] = cond ? -vi : vj;
    }
}

__device__ __forceinline__ void qrRotate(float* B, float* U, int p, int q) {
    const float eps = 1e-6f;
    float a1 = B[3 * p + p], a2 = B[3 * q + p];
    float rho2 = fmaf(a1, a1, a2 * a2);
    float rho = sqrtf(rho2);
    float sh = rho > eps ? a2 : 0.0f;
    float ch = fabsf(a1) + fmaxf(rho, eps);
    bool neg = a1 < 0.0f;
    float t = ch;
    ch = neg ? sh : ch;
    sh = neg ? t : sh;
    float w = rsqrtf(fmaf(ch, ch, sh * sh));
    ch *= w;
    sh *= w;
    float c = fmaf(ch, ch, -sh * sh);
    float s = 2.0f * ch * sh;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float bp = B[3 * p + k], bq = B[3 * q + k];
        B[3 * p + k] = fmaf(c, bp, s * bq);
        B[3 * q + k] = fmaf(-s, bp, c * bq);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float up = U[3 * k + p], uq = U[3 * k + q];
        U[3 * k + p] = fmaf(c, up, s * uq);
        U[3 * k + q] = fmaf(-s, up, c * uq);
    }
}

__device__ __forceinline__ void svd3(const float* A, float* U, float* s, float* V) {
    float S[3][3];  // A^T A (symmetric: upper triangle formed, mirrored)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
            S[i][j] = S[j][i] = fmaf(A[6 + i], A[6 + j], fmaf(A[3 + i], A[3 + j], A[i] * A[j]));
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k] = (k % 4 == 0) ? 1.0f : 0.0f;
#pragma unroll 1
    for (int sweep = 0; sweep < kSvdSweeps; ++sweep) {
        jacobiRotate(S, V, 0, 1);
        jacobiRotate(S, V, 1, 2);
        jacobiRotate(S, V, 0, 2);
    }
    float B[9];
    matmul3(A, V, B);
    float r0 = fmaf(B[6], B[6], fmaf(B[3], B[3], B[0] * B[0]));
    float r1 = fmaf(B[7], B[7], fmaf(B[4], B[4], B[1] * B[1]));
    float r2 = fmaf(B[8], B[8], fmaf(B[5], B[5], B[2] * B[2]));
    bool c01 = r0 < r1;
    condSwapNeg(c01, B, V, 0, 1);
    float t = r0;
    r0 = c01 ? r1 : r0;
    r1 = c01 ? t : r1;
    bool c02 = r0 < r2;
    condSwapNeg(c02, B, V, 0, 2);
    t = r0;
    r0 = c02 ? r2 : r0;
    r2 = c02 ? t : r2;
    bool c12 = r1 < r2;
    condSwapNeg(c12, B, V, 1, 2);
#pragma unroll
    for (int k = 0; k < 9; ++k) U[k] = (k % 4 == 0) ? 1.0f : 0.0f;
    qrRotate(B, U, 0, 1);
    qrRotate(B, U, 0, 2);
    qrRotate(B, U, 1, 2);
    s[0] = B[0];
    s[1] = B[4];
    s[2] = B[8];
}

// ---------------------------------------------------------------------------
// Elastic fast path of the plasticity update.  When no singular value of F
// leaves (lo, hi), the clamp changes nothing (Fe = F, Fp unchanged) and the
// stress needs only F and its rotation R = U V^T:
//   fixed corotated  2 mu U diag(s (s - 1)) U^T = 2 mu (F - R) F^T,
//   Neo-Hookean      mu U diag(s^2) U^T        = mu F F^T.
// ---------------------------------------------------------------------------
// Whether det F > 0 and every singular value of F lies strictly inside
// (lo, hi): hi^2 I - F^T F and F^T F - lo^2 I both positive definite (leading
// principal minors > 0, Sylvester).  A case this FP32 test cannot decide
// (a singular value within rounding of a bound) reports false, and the
// caller takes the SVD path, which clamps exactly.
__device__ __forceinline__ bool singularValuesInside(const float* F, float lo, float hi) {
    float c[3][3];  // F^T F
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) c[i][j] = c[j][i] = fmaf(F[6 + i], F[6 + j], fmaf(F[3 + i], F[3 + j], F[i] * F[j]));
    auto pd = [](float a00, float a11, float a22, float a01, float a02, float a12) {
        const float m2 = fmaf(a00, a11, -a01 * a01);
        const float d = a00 * fmaf(a11, a22, -a12 * a12) - a01 * fmaf(a01, a22, -a12 * a02) +
                        a02 * fmaf(a01, a12, -a11 * a02);
        return a00 > 0.f && m2 > 0.f && d > 0.f;
    };
    const float h2 = hi * hi, l2 = lo * lo;
    return det3(F) > 0.f && pd(h2 - c[0][0], h2 - c[1][1], h2 - c[2][2], -c[0][1], -c[0][2], -c[1][2]) &&
           pd(c[0][0] - l2, c[1][1] - l2, c[2][2] - l2, c[0][1], c[0][2], c[1][2]);
}

// Rotation of the polar decomposition F = R S by Newton's iteration
// R <- (R + R^-T) / 2 from R = F (quadratic convergence; with every singular
// value within 10 % of 1, three steps reach FP32 round-off, four within 25 %).
// R^-T = cof(R) / det R.
__device__ __forceinline__ void polarRotation(const float* F, float* R, int iterations) {
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] = F[k];
#pragma unroll 1
    for (int it = 0; it < iterations; ++it) {
        float c[9];
        c[0] = fmaf(R[4], R[8], -R[5] * R[7]);
        c[1] = fmaf(R[5], R[6], -R[3] * R[8]);
        c[2] = fmaf(R[3], R[7], -R[4] * R[6]);
        c[3] = fmaf(R[2], R[7], -R[1] * R[8]);
        c[4] = fmaf(R[0], R[8], -R[2] * R[6]);
        c[5] = fmaf(R[1], R[6], -R[0] * R[7]);
        c[6] = fmaf(R[1], R[5], -R[2] * R[4]);
        c[7] = fmaf(R[2], R[3], -R[0] * R[5]);
        c[8] = fmaf(R[0], R[4], -R[1] * R[3]);
        const float det = fmaf(R[0], c[0], fmaf(R[1], c[1], R[2] * c[2]));
        const float h = 0.5f / det;
#pragma unroll
        for (int k = 0; k < 9; ++k) R[k] = fmaf(h, c[k], 0.5f * R[k]);
    }
}

// ---------------------------------------------------------------------------
// applyBoundaryCollision (src/collision_object3d.cu:7-54).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void boundaryCollision(const float* pos, float* vel, const float* lo, const float* hi,
                                                  float friction) {
    float n[3] = {0.f, 0.f, 0.f};
    bool collided = false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (pos[i] <= lo[i] + kFltEps) {
            collided = true;
            n[i] = 1.0f;
        }
        if (pos[i] >= hi[i] - kFltEps) {
            collided = true;
            n[i] = -1.0f;
        }
    }
    if (!collided) return;
    float vn = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2];
    if (vn >= kFltEps) return;
    float vt[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) vt[i] = vel[i] - vn * n[i];
    float vtn = sqrtf(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
    if (vtn <= -friction * vn + kFltEps) {
        vel[0] = vel[1] = vel[2] = 0.0f;
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) vel[i] = vt[i] + friction * vn * (vt[i] / vtn);
    }
}

}  // namespace mpm
