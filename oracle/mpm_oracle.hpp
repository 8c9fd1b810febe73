// mpm_oracle.hpp -- CPU restatement of the H-YWu/mpm particle step.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py may load this code.  The
// product (mpm_b200/) never links or calls it.
//
// Parity unpinned: the reference cannot be compiled in this environment
// (Eigen 3.4 and yaml-cpp are fetched at configure time, the
// external/3x3_SVD_CUDA submodule is empty, and the material/SVD functions are
// __device__-only), and the reference ships no tests or golden vectors.  This
// restatement is pinned instead by known-answer tests derived from the
// mathematics the reference implements (partition of unity, APIC inertia
// tensors, SVD reconstruction, collision cases, ...; tests/test_oracle.py) and
// by agreement between its FP32 and FP64 instantiations.
//
// Two instantiations:
//   Real = float : "reference restatement" -- the reference's operation order,
//                  float storage and double-literal intermediates;
//                  3x3 SVD by the McAdams et al. 2011 approximate-Givens
//                  Jacobi method (the algorithm of the reference's
//                  un-vendored 3x3_SVD_CUDA dependency), 4 sweeps.
//   Real = double: FP64 oracle -- same step, every intermediate in double and
//                  an exact cyclic-Jacobi SVD run to convergence.
//
// Each function cites the reference file:line it follows.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "../include/mpm_b200.h"

namespace oracle {

constexpr float kFltEps = std::numeric_limits<float>::epsilon();

template <class R>
struct Vec3 {
    R v[3];
    R& operator[](int i) { return v[i]; }
    const R& operator[](int i) const { return v[i]; }
};

// Row-major 3x3.
template <class R>
struct Mat3 {
    R a[9];
    R& operator()(int i, int j) { return a[3 * i + j]; }
    const R& operator()(int i, int j) const { return a[3 * i + j]; }
    static Mat3 identity() {
        Mat3 m{};
        m(0, 0) = m(1, 1) = m(2, 2) = R(1);
        return m;
    }
    static Mat3 zero() { return Mat3{}; }
};

template <class R>
inline Mat3<R> matmul(const Mat3<R>& A, const Mat3<R>& B) {
    Mat3<R> C{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            R s = A(i, 0) * B(0, j);
            s = s + A(i, 1) * B(1, j);
            s = s + A(i, 2) * B(2, j);
            C(i, j) = s;
        }
    return C;
}

template <class R>
inline Mat3<R> transpose(const Mat3<R>& A) {
    Mat3<R> T{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T(i, j) = A(j, i);
    return T;
}

// Cofactor expansion along the first row.
template <class R>
inline R det3(const Mat3<R>& m) {
    return m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) -
           m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
           m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
}

// ---------------------------------------------------------------------------
// Interpolation kernels: src/interpolation3d.cu:88-142.  The reference
// writes double literals, so for Real = float the 1D kernel is evaluated in
// double (with float products where the reference multiplies two floats) and
// rounded to float on return.
// ---------------------------------------------------------------------------
template <class R>
inline R linearN(R x) {  // :88-93
    R xabs = std::fabs(x);
    if (xabs < 1.0) return (R)(1.0 - xabs);
    return (R)0.0;
}
template <class R>
inline R linearNDot(R x) {  // :96-102
    R xabs = std::fabs(x);
    if (xabs < 1.0 && xabs > (R)kFltEps) return -x / xabs;
    return (R)0.0;
}
template <class R>
inline R quadraticN(R x) {  // :105-112
    R xabs = std::fabs(x);
    if (xabs < 0.5) return (R)(0.75 - (R)(xabs * xabs));
    if (xabs < 1.5) return (R)(0.5 * std::pow(1.5 - (double)xabs, 2));
    return (R)0.0;
}
template <class R>
inline R quadraticNDot(R x) {  // :115-122
    R xabs = std::fabs(x);
    if (xabs < 0.5) return (R)(-2.0 * (double)x);
    if (xabs < 1.5) return (R)(-(1.5 * (double)x / (double)xabs) + (double)x);
    return (R)0.0;
}
template <class R>
inline R cubicN(R x) {  // :125-132
    R xabs = std::fabs(x);
    if (xabs < 1.0)
        return (R)(0.5 * std::pow((double)xabs, 3) - (double)(R)(xabs * xabs) + 2.0 / 3.0);
    if (xabs < 2.0) return (R)(std::pow(2.0 - (double)xabs, 3) / 6.0);
    return (R)0.0;
}
template <class R>
inline R cubicNDot(R x) {  // :135-142
    R xabs = std::fabs(x);
    if (xabs < 1.0) return (R)(1.5 * (double)x * (double)xabs - 2.0 * (double)x);
    if (xabs < 2.0)
        return (R)(-(2.0 * (double)x / (double)xabs) + 2.0 * (double)x -
                   0.5 * (double)(R)(x * xabs));
    return (R)0.0;
}

template <class R>
inline R splineN(int type, R x) {
    switch (type) {
        case MPM_INTERP_LINEAR: return linearN(x);
        case MPM_INTERP_QUADRATIC_BSPLINE: return quadraticN(x);
        default: return cubicN(x);
    }
}
template <class R>
inline R splineNDot(int type, R x) {
    switch (type) {
        case MPM_INTERP_LINEAR: return linearNDot(x);
        case MPM_INTERP_QUADRATIC_BSPLINE: return quadraticNDot(x);
        default: return cubicNDot(x);
    }
}
// Interpolator3D::setRange (src/interpolation3d.cu:69-85).
inline float splineRange(int type) {
    switch (type) {
        case MPM_INTERP_LINEAR: return 1.0f;
        case MPM_INTERP_QUADRATIC_BSPLINE: return 1.5f;
        default: return 2.0f;
    }
}

// weight3D / weightGradient3D (src/interpolation3d.cu:14-66).
template <class R>
inline R weight3D(int type, const Vec3<R>& xp, const Vec3<R>& xi, R h) {
    R x = (xp[0] - xi[0]) / h, y = (xp[1] - xi[1]) / h, z = (xp[2] - xi[2]) / h;
    return splineN(type, x) * splineN(type, y) * splineN(type, z);
}
template <class R>
inline Vec3<R> weightGradient3D(int type, const Vec3<R>& xp, const Vec3<R>& xi, R h) {
    R x = (xp[0] - xi[0]) / h, y = (xp[1] - xi[1]) / h, z = (xp[2] - xi[2]) / h;
    Vec3<R> g;
    g[0] = (splineNDot(type, x) * splineN(type, y) * splineN(type, z)) / h;
    g[1] = (splineN(type, x) * splineNDot(type, y) * splineN(type, z)) / h;
    g[2] = (splineN(type, x) * splineN(type, y) * splineNDot(type, z)) / h;
    return g;
}

// ---------------------------------------------------------------------------
// 3x3 SVD.  Output convention of the reference's svd3x3 (src/svd_eigen.cu:7-17):
// A = U diag(s) V^T, U and V proper rotations, s sorted by decreasing
// magnitude, s[2] carries the sign of det(A).
// ---------------------------------------------------------------------------

// McAdams, Selle, Tamstorf, Teran, Sifakis, "Computing the Singular Value
// Decomposition of 3x3 matrices with minimal branching and elementary
// floating point operations", UW-Madison CS TR-1690 (2011): Jacobi
// eigen-analysis of A^T A with approximate Givens rotations, a sort of the
// columns of A V with sign fixes, and a Givens QR of A V.
template <class R>
void svdMcAdams(const Mat3<R>& A, Mat3<R>& U, Vec3<R>& s, Mat3<R>& V, int sweeps = 4);

// Exact cyclic Jacobi (to convergence) for the FP64 oracle.
void svdExact(const Mat3<double>& A, Mat3<double>& U, Vec3<double>& s, Mat3<double>& V);

template <class R>
inline void svd3(const Mat3<R>& A, Mat3<R>& U, Vec3<R>& s, Mat3<R>& V);
template <>
inline void svd3<float>(const Mat3<float>& A, Mat3<float>& U, Vec3<float>& s, Mat3<float>& V) {
    svdMcAdams<float>(A, U, s, V, 4);
}
template <>
inline void svd3<double>(const Mat3<double>& A, Mat3<double>& U, Vec3<double>& s, Mat3<double>& V) {
    svdExact(A, U, s, V);
}

// applyBoundaryCollision (src/collision_object3d.cu:7-54).
template <class R>
Vec3<R> applyBoundaryCollision(const Vec3<R>& position, const Vec3<R>& velocity,
                               const Vec3<R>& grid000, const Vec3<R>& grid111, R friction);

// ---------------------------------------------------------------------------
// Particle and grid state (include/material_point3d.h:14-22,
// include/apic_material_point3d.h:14-23, include/grid3d.h:9-35).
// ---------------------------------------------------------------------------
template <class R>
struct Particle {
    R volume0, mass;
    Vec3<R> x, v;
    Mat3<R> Fe, Fp;
    R mu0, lambda0, xi, theta_c, theta_s;
    int model;
    Mat3<R> B;  // APIC only
};

template <class R>
struct Node {
    Vec3<R> force, velocity, velocity_star;
    R mass;
};

template <class R>
class Solver {
public:
    using Real = R;
    Solver(const mpm_scene_desc& d, const mpm_particles_in& in);

    void initialize();                 // src/mpm_solver3d.cu:131-223
    void resetGrid();                  // :225-235
    void particlesToGrid();            // :237-294 / apic :245-304
    void computeGravityForces();       // :394-403
    void updateGridVelocities(R dt);   // :300-310
    void gridCollision(R dt);          // :405-426
    void gridToParticles(R dt, R blend);  // :316-379 / apic :326-388
    void particlesCollision(R dt);     // :428-445
    void advectParticles(R dt);        // :381-391
    void solveLinearSystem(R dt);      // :312-314 (a TODO there): semi-implicit solve
    // H u: the elastic Hessian applied to node velocities u (zero at massless
    // nodes), out = sum_p V0 (dP/dF : (sum_j u_j grad w_jp^T) Fe) Fe^T grad w_ip
    void hessianAction(const std::vector<Vec3<R>>& u, std::vector<Vec3<R>>& out);
    // grid force -sum_p V0 P(F^) Fe^T grad w_ip with F^ = (I + sum_j d_j grad w_jp^T) Fe
    // (nodes displaced by d): finite differences of it check hessianAction
    void displacedForce(const std::vector<Vec3<R>>& d, std::vector<Vec3<R>>& out);
    void simulateOneStep();            // :100-125

    mpm_scene_desc desc;
    bool enable_particles_collision = false;
    int threads = 1;
    std::vector<Particle<R>> particles;
    std::vector<Node<R>> grid;
    Vec3<R> origin, target;
    R h;
    int res[3];
    R Dinv = 0;  // APIC: (k h^2)^-1, src/apic_mpm_solver3d.cu:151-157
    // Level-set collision object (include/collision_object3d.h:9-12): signed
    // distance per node, negative inside; applied after the grid boundary.
    // semi-implicit update (beta > 0): (M + beta dt^2 H) v = M v*, conjugate
    // residual to |r| <= tol |M v*| or max_iter iterations
    R beta = 0;
    int max_iter = 30;
    R tol = (R)1e-5;
    int last_iters = 0;
    double last_residual = 0;
    // CFL time step: cfl > 0 makes each step's dt min(desc.dt, cfl h / max|v_p|)
    R cfl = 0;
    double time = 0;
    R last_dt = 0;
    bool has_phi = false;
    std::vector<R> phi;
    R phi_friction = 0;
    Vec3<R> phi_vel{};

private:
    void stencilRange(const Vec3<R>& x, int lo[3], int hi[3]) const;
    template <class F>
    void forEachNode(const Particle<R>& p, F&& f) const;
    template <class Body>
    void scatterDeterministic(Body&& body);
};

}  // namespace oracle
