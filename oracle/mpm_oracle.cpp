// mpm_oracle.cpp -- CPU restatement of the H-YWu/mpm particle step.
// TEST INFRASTRUCTURE ONLY (see mpm_oracle.hpp).  Parity unpinned against an
// executed reference: the reference does not build here; pinned by
// known-answer tests instead.
#include "mpm_oracle.hpp"

#include <algorithm>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

// ---------------------------------------------------------------------------
// SVD, McAdams et al. 2011 (approximate Givens Jacobi + sorted Givens QR).
// ---------------------------------------------------------------------------
namespace {

template <class R>
struct Sym3 {  // symmetric matrix, full storage
    R m[3][3];
};

// Approximate Givens half-angle (cos(t/2), sin(t/2)) that (nearly)
// annihilates the off-diagonal of the 2x2 block [[app, apq],[apq, aqq]].
// Falls back to t/2 = pi/8 when the first-order estimate would exceed it.
template <class R>
inline void approxGivens(R app, R apq, R aqq, R& ch, R& sh) {
    const R gamma = (R)5.82842712474619009760;  // 3 + 2 sqrt(2) = cot^2(pi/8)
    const R cstar = (R)0.92387953251128675613;  // cos(pi/8)
    const R sstar = (R)0.38268343236508977173;  // sin(pi/8)
    ch = (R)2 * (app - aqq);
    sh = apq;
    if (gamma * sh * sh < ch * ch) {
        R w = (R)1 / std::sqrt(ch * ch + sh * sh);
        ch *= w;
        sh *= w;
    } else {
        ch = cstar;
        sh = sstar;
    }
}

// Conjugate S by the rotation G acting in the (p,q) plane:  S <- G^T S G,
// V <- V G, with G = [[c, -s],[s, c]] on coordinates (p, q).
template <class R>
inline void rotateSym(Sym3<R>& S, Mat3<R>& V, int p, int q, R c, R s) {
    for (int k = 0; k < 3; ++k) {  // columns: S <- S G
        R sp = S.m[k][p], sq = S.m[k][q];
        S.m[k][p] = c * sp + s * sq;
        S.m[k][q] = -s * sp + c * sq;
    }
    for (int k = 0; k < 3; ++k) {  // rows: S <- G^T S
        R sp = S.m[p][k], sq = S.m[q][k];
        S.m[p][k] = c * sp + s * sq;
        S.m[q][k] = -s * sp + c * sq;
    }
    for (int k = 0; k < 3; ++k) {
        R vp = V(k, p), vq = V(k, q);
        V(k, p) = c * vp + s * vq;
        V(k, q) = -s * vp + c * vq;
    }
}

template <class R>
inline void swapCols(Mat3<R>& M, int i, int j, bool negate_j) {
    for (int k = 0; k < 3; ++k) {
        R t = M(k, i);
        M(k, i) = M(k, j);
        M(k, j) = negate_j ? -t : t;
    }
}

// Sort the columns of B (and V) by decreasing squared norm; every swap
// negates one column so that det(V) stays +1.
template <class R>
inline void sortColumns(Mat3<R>& B, Mat3<R>& V) {
    auto n2 = [&](int j) { return B(0, j) * B(0, j) + B(1, j) * B(1, j) + B(2, j) * B(2, j); };
    R r0 = n2(0), r1 = n2(1), r2 = n2(2);
    if (r0 < r1) {
        swapCols(B, 0, 1, true);
        swapCols(V, 0, 1, true);
        std::swap(r0, r1);
    }
    if (r0 < r2) {
        swapCols(B, 0, 2, true);
        swapCols(V, 0, 2, true);
        std::swap(r0, r2);
    }
    if (r1 < r2) {
        swapCols(B, 1, 2, true);
        swapCols(V, 1, 2, true);
        std::swap(r1, r2);
    }
}

// Apply a Givens rotation to rows (p,q) of B (B <- G^T B) and columns (p,q)
// of U (U <- U G).
template <class R>
inline void rotateRows(Mat3<R>& B, Mat3<R>& U, int p, int q, R c, R s) {
    for (int k = 0; k < 3; ++k) {
        R bp = B(p, k), bq = B(q, k);
        B(p, k) = c * bp + s * bq;
        B(q, k) = -s * bp + c * bq;
    }
    for (int k = 0; k < 3; ++k) {
        R up = U(k, p), uq = U(k, q);
        U(k, p) = c * up + s * uq;
        U(k, q) = -s * up + c * uq;
    }
}

// Half-angle QR Givens of McAdams et al.: maps (a1, a2) to (+rho, 0).
template <class R>
inline void qrGivens(R a1, R a2, R& c, R& s) {
    const R eps = (R)1e-6;
    R rho = std::sqrt(a1 * a1 + a2 * a2);
    R sh = rho > eps ? a2 : (R)0;
    R ch = std::fabs(a1) + std::max(rho, eps);
    if (a1 < 0) std::swap(ch, sh);
    R w = (R)1 / std::sqrt(ch * ch + sh * sh);
    ch *= w;
    sh *= w;
    c = ch * ch - sh * sh;
    s = (R)2 * ch * sh;
}

}  // namespace

template <class R>
void svdMcAdams(const Mat3<R>& A, Mat3<R>& U, Vec3<R>& s, Mat3<R>& V, int sweeps) {
    Mat3<R> At = transpose(A);
    Mat3<R> AtA = matmul(At, A);
    Sym3<R> S;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S.m[i][j] = AtA(i, j);
    V = Mat3<R>::identity();
    static const int P[3] = {0, 1, 0}, Q[3] = {1, 2, 2};
    for (int sw = 0; sw < sweeps; ++sw) {
        for (int k = 0; k < 3; ++k) {
            int p = P[k], q = Q[k];
            R ch, sh;
            approxGivens(S.m[p][p], S.m[p][q], S.m[q][q], ch, sh);
            R c = ch * ch - sh * sh, sn = (R)2 * ch * sh;
            rotateSym(S, V, p, q, c, sn);
        }
    }
    Mat3<R> B = matmul(A, V);
    sortColumns(B, V);
    U = Mat3<R>::identity();
    R c, sn;
    qrGivens(B(0, 0), B(1, 0), c, sn);
    rotateRows(B, U, 0, 1, c, sn);
    qrGivens(B(0, 0), B(2, 0), c, sn);
    rotateRows(B, U, 0, 2, c, sn);
    qrGivens(B(1, 1), B(2, 1), c, sn);
    rotateRows(B, U, 1, 2, c, sn);
    s[0] = B(0, 0);
    s[1] = B(1, 1);
    s[2] = B(2, 2);
}

template void svdMcAdams<float>(const Mat3<float>&, Mat3<float>&, Vec3<float>&, Mat3<float>&, int);
template void svdMcAdams<double>(const Mat3<double>&, Mat3<double>&, Vec3<double>&, Mat3<double>&, int);

void svdExact(const Mat3<double>& A, Mat3<double>& U, Vec3<double>& s, Mat3<double>& V) {
    Mat3<double> AtA = matmul(transpose(A), A);
    Sym3<double> S;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S.m[i][j] = AtA(i, j);
    V = Mat3<double>::identity();
    static const int P[3] = {0, 1, 0}, Q[3] = {1, 2, 2};
    for (int sw = 0; sw < 60; ++sw) {
        double off = S.m[0][1] * S.m[0][1] + S.m[1][2] * S.m[1][2] + S.m[0][2] * S.m[0][2];
        double dia = S.m[0][0] * S.m[0][0] + S.m[1][1] * S.m[1][1] + S.m[2][2] * S.m[2][2];
        if (off <= 1e-34 * dia || off == 0.0) break;
        for (int k = 0; k < 3; ++k) {
            int p = P[k], q = Q[k];
            double apq = S.m[p][q];
            if (apq == 0.0) continue;
            // Classic Jacobi: tau = (aqq - app) / (2 apq), t = sign(tau)/(|tau| + sqrt(1+tau^2)).
            double tau = (S.m[q][q] - S.m[p][p]) / (2.0 * apq);
            double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
            double c = 1.0 / std::sqrt(1.0 + t * t), sn = t * c;
            // rotateSym uses G = [[c,-s],[s,c]]; the Jacobi rotation that zeroes
            // apq with this t is G = [[c, s],[-s, c]], i.e. angle -theta.
            rotateSym(S, V, p, q, c, -sn);
        }
    }
    Mat3<double> B = matmul(A, V);
    sortColumns(B, V);
    U = Mat3<double>::identity();
    auto exactGivens = [](double a1, double a2, double& c, double& sn) {
        double rho = std::hypot(a1, a2);
        if (rho == 0.0) {
            c = 1.0;
            sn = 0.0;
        } else {
            c = a1 / rho;
            sn = a2 / rho;
        }
    };
    double c, sn;
    exactGivens(B(0, 0), B(1, 0), c, sn);
    rotateRows(B, U, 0, 1, c, sn);
    exactGivens(B(0, 0), B(2, 0), c, sn);
    rotateRows(B, U, 0, 2, c, sn);
    exactGivens(B(1, 1), B(2, 1), c, sn);
    rotateRows(B, U, 1, 2, c, sn);
    s[0] = B(0, 0);
    s[1] = B(1, 1);
    s[2] = B(2, 2);
}

// ---------------------------------------------------------------------------
// Boundary collision: src/collision_object3d.cu:7-54.
// ---------------------------------------------------------------------------
template <class R>
Vec3<R> applyBoundaryCollision(const Vec3<R>& position, const Vec3<R>& velocity,
                               const Vec3<R>& grid000, const Vec3<R>& grid111, R friction) {
    const R eps = (R)kFltEps;
    Vec3<R> updated = velocity, rel = velocity, normal{};
    bool collided = false;
    for (int i = 0; i < 3; ++i) {  // :20-29
        if (position[i] <= grid000[i] + eps) {
            collided = true;
            normal[i] = (R)1.0;
        }
        if (position[i] >= grid111[i] - eps) {
            collided = true;
            normal[i] = (R)-1.0;
        }
    }
    if (collided) {  // :31-51
        R vn = rel[0] * normal[0] + rel[1] * normal[1] + rel[2] * normal[2];
        if (vn >= eps) return updated;
        Vec3<R> vt;
        for (int i = 0; i < 3; ++i) vt[i] = rel[i] - vn * normal[i];
        R vtn = std::sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
        if (vtn <= -friction * vn + eps) {
            rel = Vec3<R>{};
        } else {
            for (int i = 0; i < 3; ++i) rel[i] = vt[i] + friction * vn * (vt[i] / vtn);
        }
        updated = rel;
    }
    return updated;
}

// Level-set collision object: trilinear signed distance and gradient at
// pos (clamped to the grid); where the distance is <= 0 the friction law of
// applyBoundaryCollision (src/collision_object3d.cu:38-51) acts on the
// velocity relative to the object's surface velocity, normal = normalised
// gradient.  The reference declares LevelSetCollisionObject3D
// (include/collision_object3d.h:9-12) but never applies it.
template <class R>
Vec3<R> applyLevelSetCollision(const Vec3<R>& pos, const Vec3<R>& vel, const R* phi, const int res[3],
                               const Vec3<R>& origin, R h, R friction, const Vec3<R>& vco) {
    const R eps = (R)kFltEps;
    int i0[3];
    R f[3];
    const R inv_h = (R)1 / h;
    for (int a = 0; a < 3; ++a) {
        R g = (pos[a] - origin[a]) * inv_h;
        g = std::min(std::max(g, (R)0), (R)(res[a] - 1));
        i0[a] = std::min((int)g, res[a] - 2);
        f[a] = g - (R)i0[a];
    }
    const size_t X = (size_t)res[0], XY = X * (size_t)res[1];
    R val = 0, gr[3] = {0, 0, 0};
    for (int k = 0; k < 8; ++k) {
        const int d[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
        const R c = phi[(size_t)(i0[0] + d[0]) + X * (size_t)(i0[1] + d[1]) + XY * (size_t)(i0[2] + d[2])];
        R w[3], sg[3];
        for (int a = 0; a < 3; ++a) {
            w[a] = d[a] ? f[a] : (R)1 - f[a];
            sg[a] = d[a] ? (R)1 : (R)-1;
        }
        val += c * (w[0] * w[1] * w[2]);
        gr[0] += c * (sg[0] * w[1] * w[2]);
        gr[1] += c * (w[0] * sg[1] * w[2]);
        gr[2] += c * (w[0] * w[1] * sg[2]);
    }
    if (val > 0) return vel;
    const R gn = std::sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
    if (!(gn > 0)) return vel;
    Vec3<R> n, rel, out;
    for (int a = 0; a < 3; ++a) {
        n[a] = gr[a] / gn;
        rel[a] = vel[a] - vco[a];
    }
    const R vn = rel[0] * n[0] + rel[1] * n[1] + rel[2] * n[2];
    if (vn >= eps) return vel;
    Vec3<R> vt;
    for (int a = 0; a < 3; ++a) vt[a] = rel[a] - vn * n[a];
    const R vtn = std::sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
    if (vtn <= -friction * vn + eps) return vco;
    for (int a = 0; a < 3; ++a) out[a] = (vt[a] + friction * vn * (vt[a] / vtn)) + vco[a];
    return out;
}

template Vec3<float> applyBoundaryCollision(const Vec3<float>&, const Vec3<float>&, const Vec3<float>&,
                                            const Vec3<float>&, float);
template Vec3<double> applyBoundaryCollision(const Vec3<double>&, const Vec3<double>&,
                                             const Vec3<double>&, const Vec3<double>&, double);

// ---------------------------------------------------------------------------
// Material point: src/material_point3d.cu.
// ---------------------------------------------------------------------------
namespace {

// plasticLame (src/material_point3d.cu:158-162).  The reference stores the
// decaying factor in a float before multiplying.
template <class R>
inline void plasticLame(const Particle<R>& p, R& mu, R& la) {
    R Jp = det3(p.Fp);
    R f = (R)std::exp((double)p.xi * (1.0 - (double)Jp));
    mu = p.mu0 * f;
    la = p.lambda0 * f;
}

// fixedCorotated...Transpose (:110-128): 2 mu (Fe - R) Fe^T + la (Je-1) Je I.
template <class R>
inline Mat3<R> fcrStress(const Particle<R>& p) {
    R mu, la;
    plasticLame(p, mu, la);
    Mat3<R> U, V;
    Vec3<R> s;
    svd3(p.Fe, U, s, V);
    Mat3<R> Rm = matmul(U, transpose(V));
    R Je = det3(p.Fe);
    Mat3<R> D{};
    for (int i = 0; i < 9; ++i) D.a[i] = p.Fe.a[i] - Rm.a[i];
    Mat3<R> P = matmul(D, transpose(p.Fe));
    R two_mu = (R)(2.0 * (double)mu);
    R lj = (R)((double)la * ((double)Je - 1.0) * (double)Je);
    for (int i = 0; i < 9; ++i) P.a[i] = two_mu * P.a[i];
    for (int i = 0; i < 3; ++i) P(i, i) += lj;
    return P;
}

// NeoHookean...Transpose (:131-155).  Projects Fe (writes it back) so that
// its singular values are >= FLT_EPSILON.
template <class R>
inline Mat3<R> nhStress(Particle<R>& p) {
    R mu, la;
    plasticLame(p, mu, la);
    Mat3<R> U, V;
    Vec3<R> s;
    svd3(p.Fe, U, s, V);
    for (int i = 0; i < 3; ++i) s[i] = std::max(s[i], (R)kFltEps);
    Mat3<R> S{};
    for (int i = 0; i < 3; ++i) S(i, i) = s[i];
    p.Fe = matmul(matmul(U, S), transpose(V));
    R Je = det3(p.Fe);
    Mat3<R> P = matmul(p.Fe, transpose(p.Fe));
    for (int i = 0; i < 9; ++i) P.a[i] = mu * P.a[i];
    R l = (R)((double)la * std::log((double)Je));
    for (int i = 0; i < 3; ++i) P(i, i) += l - mu;
    return P;
}

// volumeTimesCauchyStress (:33-45).
template <class R>
inline Mat3<R> volumeTimesCauchyStress(Particle<R>& p) {
    Mat3<R> P = (p.model == MPM_MODEL_NEO_HOOKEAN) ? nhStress(p) : fcrStress(p);
    for (int i = 0; i < 9; ++i) P.a[i] = p.volume0 * P.a[i];
    return P;
}

// Cofactor matrix J F^-T of a 3x3 matrix by columns: c0 = f1 x f2,
// c1 = f2 x f0, c2 = f0 x f1 (f_k = column k).
template <class R>
inline Vec3<R> cross3(const Vec3<R>& a, const Vec3<R>& b) {
    return Vec3<R>{{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
}
template <class R>
inline Vec3<R> column(const Mat3<R>& A, int k) {
    return Vec3<R>{{A(0, k), A(1, k), A(2, k)}};
}
template <class R>
inline Mat3<R> cofactor(const Mat3<R>& F) {
    Mat3<R> C{};
    for (int k = 0; k < 3; ++k) {
        Vec3<R> c = cross3(column(F, (k + 1) % 3), column(F, (k + 2) % 3));
        for (int r = 0; r < 3; ++r) C(r, k) = c[r];
    }
    return C;
}
// Differential of the cofactor along dF (linear in dF).
template <class R>
inline Mat3<R> cofactorDifferential(const Mat3<R>& F, const Mat3<R>& dF) {
    Mat3<R> C{};
    for (int k = 0; k < 3; ++k) {
        const int a = (k + 1) % 3, b = (k + 2) % 3;
        Vec3<R> c1 = cross3(column(dF, a), column(F, b)), c2 = cross3(column(F, a), column(dF, b));
        for (int r = 0; r < 3; ++r) C(r, k) = c1[r] + c2[r];
    }
    return C;
}

// dP/dF : dF at Fe for the first Piola stress P of the two models (the
// stresses above are P Fe^T).  Fixed corotated: P = 2 mu (F - R) + la (J - 1)
// cof F, dP = 2 mu (dF - dR) + la (dJ cof F + (J - 1) dcof F) with
// dR = U W V^T, W_ij = (M_ij - M_ji) / (s_i + s_j), M = U^T dF V (the
// rotation differential of the polar decomposition; Stomakhin et al. 2013,
// "A material point method for snow simulation", supplementary notes).
// Neo-Hookean: P = mu (F - F^-T) + la ln J F^-T,
// dP = mu dF + (la ln J - mu) d(F^-T) + la (F^-T : dF) F^-T with
// d(F^-T) = -F^-T dF^T F^-T.  mu, la are the hardened Lame parameters of Fp.
template <class R>
inline Mat3<R> stressDifferential(const Particle<R>& p, const Mat3<R>& dF) {
    R mu, la;
    plasticLame(p, mu, la);
    const Mat3<R>& F = p.Fe;
    const Mat3<R> C = cofactor(F);
    const R J = det3(F);
    Mat3<R> dP{};
    if (p.model == MPM_MODEL_NEO_HOOKEAN) {
        Mat3<R> FiT{};
        for (int i = 0; i < 9; ++i) FiT.a[i] = C.a[i] / J;
        Mat3<R> dFiT = matmul(matmul(FiT, transpose(dF)), FiT);
        R dlnJ = 0;
        for (int i = 0; i < 9; ++i) dlnJ += FiT.a[i] * dF.a[i];
        const R lnJ = (R)std::log((double)J);
        for (int i = 0; i < 9; ++i) dP.a[i] = mu * dF.a[i] - (la * lnJ - mu) * dFiT.a[i] + la * dlnJ * FiT.a[i];
        return dP;
    }
    Mat3<R> U, V;
    Vec3<R> s;
    svd3(F, U, s, V);
    const Mat3<R> M = matmul(matmul(transpose(U), dF), V);
    Mat3<R> W{};
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j) {
            R den = s[i] + s[j];
            if (std::fabs(den) < (R)1e-6) den = den < 0 ? (R)-1e-6 : (R)1e-6;
            const R w = (M(i, j) - M(j, i)) / den;
            W(i, j) = w;
            W(j, i) = -w;
        }
    const Mat3<R> dR = matmul(matmul(U, W), transpose(V));
    const Mat3<R> dC = cofactorDifferential(F, dF);
    R dJ = 0;
    for (int i = 0; i < 9; ++i) dJ += C.a[i] * dF.a[i];
    for (int i = 0; i < 9; ++i)
        dP.a[i] = (R)2 * mu * (dF.a[i] - dR.a[i]) + la * (dJ * C.a[i] + (J - (R)1) * dC.a[i]);
    return dP;
}

// updateDeformationGradient (:53-70).
template <class R>
inline void updateDeformationGradient(Particle<R>& p, const Mat3<R>& gradv, R dt) {
    Mat3<R> A = Mat3<R>::identity();
    for (int i = 0; i < 9; ++i) A.a[i] += dt * gradv.a[i];
    p.Fe = matmul(A, p.Fe);
    Mat3<R> Ffull = matmul(p.Fe, p.Fp);
    Mat3<R> U, V;
    Vec3<R> s;
    svd3(p.Fe, U, s, V);
    R hi = (R)1.0 + p.theta_s, lo = (R)1.0 - p.theta_c;
    for (int i = 0; i < 3; ++i) s[i] = std::max(std::min(s[i], hi), lo);
    Mat3<R> S{}, Sinv{};
    for (int i = 0; i < 3; ++i) {
        S(i, i) = s[i];
        Sinv(i, i) = (R)1 / s[i];
    }
    p.Fe = matmul(matmul(U, S), transpose(V));
    p.Fp = matmul(matmul(matmul(V, Sinv), transpose(U)), Ffull);
}

}  // namespace

// ---------------------------------------------------------------------------
// Solver.
// ---------------------------------------------------------------------------
template <class R>
Solver<R>::Solver(const mpm_scene_desc& d, const mpm_particles_in& in) : desc(d) {
    for (int i = 0; i < 3; ++i) {
        origin[i] = (R)d.origin[i];
        res[i] = d.resolution[i];
        // Grid3DSettings: target = origin + stride * resolution (src/grid3d.cu:15)
        target[i] = (R)d.origin[i] + (R)d.stride * (R)d.resolution[i];
    }
    h = (R)d.stride;
    enable_particles_collision = d.particles_collision != 0;
    if (d.transfer == MPM_TRANSFER_APIC) {
        // src/apic_mpm_solver3d.cu:151-157 (k = 1/3 cubic, 1/4 quadratic)
        R k = 0;
        if (d.interpolation == MPM_INTERP_CUBIC_BSPLINE) k = (R)(1 / 3.0);
        if (d.interpolation == MPM_INTERP_QUADRATIC_BSPLINE) k = (R)(1 / 4.0);
        R D = k * h * h;
        Dinv = (R)1 / D;
    }
    particles.resize(in.n);
    for (size_t i = 0; i < in.n; ++i) {
        Particle<R>& p = particles[i];
        int mi = in.material ? in.material[i] : 0;
        const mpm_material& m = in.materials[mi];
        for (int a = 0; a < 3; ++a) {
            p.x[a] = (R)in.position[3 * i + a];
            p.v[a] = (R)in.velocity[3 * i + a];
        }
        p.mass = (R)in.mass[i];
        p.xi = (R)m.hardening;
        p.theta_c = (R)m.critical_compression;
        p.theta_s = (R)m.critical_stretch;
        p.model = m.model;
        // src/material_point3d.cu:25-26 (note the float product E*nu)
        double E = m.youngs_modulus, nu = m.poisson_ratio;
        p.mu0 = (R)(E / (2.0 * (1.0 + nu)));
        p.lambda0 = (R)((double)(R)((R)m.youngs_modulus * (R)m.poisson_ratio) /
                        ((1.0 + nu) * (1.0 - 2.0 * nu)));
        p.Fe = Mat3<R>::identity();
        p.Fp = Mat3<R>::identity();
        p.B = Mat3<R>::zero();
        p.volume0 = (d.volume_mode == MPM_VOLUME_PRESCRIBED && in.volume) ? (R)in.volume[i] : (R)0;
    }
    grid.assign((size_t)res[0] * res[1] * res[2], Node<R>{});
}

// Index range ceil(x/h - r) .. floor(x/h + r) (src/mpm_solver3d.cu:252-255).
template <class R>
void Solver<R>::stencilRange(const Vec3<R>& x, int lo[3], int hi[3]) const {
    R rng = (R)splineRange(desc.interpolation);
    for (int i = 0; i < 3; ++i) {
        lo[i] = (int)std::ceil(x[i] / h - rng);
        hi[i] = (int)std::floor(x[i] / h + rng);
    }
}

// The reference's triple loop with the in-grid test (src/mpm_solver3d.cu:259-264).
template <class R>
template <class F>
void Solver<R>::forEachNode(const Particle<R>& p, F&& f) const {
    int lo[3], hi[3];
    stencilRange(p.x, lo, hi);
    for (int x = lo[0]; x <= hi[0]; ++x)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int z = lo[2]; z <= hi[2]; ++z) {
                if (x < 0 || x >= res[0] || y < 0 || y >= res[1] || z < 0 || z >= res[2]) continue;
                size_t gi = (size_t)x + (size_t)res[0] * ((size_t)y + (size_t)res[1] * z);
                Vec3<R> gp;
                gp[0] = origin[0] + h * (R)x;
                gp[1] = origin[1] + h * (R)y;
                gp[2] = origin[2] + h * (R)z;
                f(gi, gp);
            }
}

// Deterministic parallel scatter: particles are bucketed by z-slab of width
// (stencil size); even slabs run in parallel, then odd slabs.  Stencils of
// same-parity slabs never overlap and each slab is walked in particle order,
// so the sums do not depend on the thread count.
template <class R>
template <class Body>
void Solver<R>::scatterDeterministic(Body&& body) {
    const int S = desc.interpolation == MPM_INTERP_LINEAR ? 2 : desc.interpolation == MPM_INTERP_QUADRATIC_BSPLINE ? 3 : 4;
    const int nslab = res[2] / S + 3;
    std::vector<int> slab(particles.size());
    std::vector<size_t> cnt(nslab + 1, 0);
    R rng = (R)splineRange(desc.interpolation);
    for (size_t i = 0; i < particles.size(); ++i) {
        R zf = std::ceil(particles[i].x[2] / h - rng);
        long long bz = std::isfinite((double)zf) ? (long long)std::max<R>(std::min<R>(zf, (R)(res[2] + 2 * S)), (R)(-2 * S)) : -2 * S;
        long long k = (bz >= 0 ? bz / S : -((-bz + S - 1) / S)) + 1;
        k = std::max<long long>(0, std::min<long long>(k, nslab - 1));
        slab[i] = (int)k;
        cnt[k + 1]++;
    }
    for (int k = 0; k < nslab; ++k) cnt[k + 1] += cnt[k];
    std::vector<size_t> order(particles.size()), fill(cnt.begin(), cnt.end() - 1);
    for (size_t i = 0; i < particles.size(); ++i) order[fill[slab[i]]++] = i;
    for (int parity = 0; parity < 2; ++parity) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
        for (int k = parity; k < nslab; k += 2)
            for (size_t j = cnt[k]; j < cnt[k + 1]; ++j) body(order[j]);
    }
}

// initialize(): P2GMass then G2PVolume (src/mpm_solver3d.cu:131-223); APIC
// variant (src/apic_mpm_solver3d.cu:130-231).  Unlike the reference, the grid
// mass is cleared first so that a repeated initialize() is idempotent.
template <class R>
void Solver<R>::initialize() {
    for (auto& n : grid) n.mass = 0;
    scatterDeterministic([&](size_t i) {
        const Particle<R>& p = particles[i];
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            R w = weight3D(desc.interpolation, p.x, gp, h);
            grid[gi].mass += p.mass * w;
        });
    });
    if (desc.volume_mode == MPM_VOLUME_PRESCRIBED) return;
    R inv_cell_vol = (R)(1.0 / (double)(h * h * h));
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long i = 0; i < (long long)particles.size(); ++i) {
        Particle<R>& p = particles[i];
        R dens = 0;
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            R w = weight3D(desc.interpolation, p.x, gp, h);
            dens += (grid[gi].mass * w) * inv_cell_vol;
        });
        p.volume0 = p.mass / dens;
    }
}

template <class R>
void Solver<R>::resetGrid() {
    for (auto& n : grid) n = Node<R>{};
}

// particlesToGrid (src/mpm_solver3d.cu:237-294; APIC src/apic_mpm_solver3d.cu:245-304).
template <class R>
void Solver<R>::particlesToGrid() {
    const bool apic = desc.transfer == MPM_TRANSFER_APIC;
    std::vector<Mat3<R>> volStress(particles.size());
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long i = 0; i < (long long)particles.size(); ++i) {
        Mat3<R> s = volumeTimesCauchyStress(particles[i]);
        for (int k = 0; k < 9; ++k) s.a[k] = -s.a[k];
        volStress[i] = s;
    }
    scatterDeterministic([&](size_t i) {
        const Particle<R>& p = particles[i];
        const Mat3<R>& vs = volStress[i];
        Mat3<R> C{};
        if (apic)
            for (int k = 0; k < 9; ++k) C.a[k] = p.B.a[k] * Dinv;  // B * Dinv, Dinv = (k h^2)^-1 I
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            R w = weight3D(desc.interpolation, p.x, gp, h);
            Vec3<R> g = weightGradient3D(desc.interpolation, p.x, gp, h);
            R m_ip = p.mass * w;
            Node<R>& n = grid[gi];
            n.mass += m_ip;
            if (apic) {
                Vec3<R> d;
                for (int a = 0; a < 3; ++a) d[a] = gp[a] - p.x[a];
                for (int a = 0; a < 3; ++a) {
                    R cd = C(a, 0) * d[0] + C(a, 1) * d[1] + C(a, 2) * d[2];
                    n.velocity[a] += m_ip * (p.v[a] + cd);
                }
            } else {
                for (int a = 0; a < 3; ++a) n.velocity[a] += p.v[a] * m_ip;
            }
            for (int a = 0; a < 3; ++a) n.force[a] += vs(a, 0) * g[0] + vs(a, 1) * g[1] + vs(a, 2) * g[2];
        });
    });
}

// computeGravityForces (src/mpm_solver3d.cu:394-403); g is 9.80665 in the reference.
template <class R>
void Solver<R>::computeGravityForces() {
    double g = desc.gravity == 9.80665f ? 9.80665 : (double)desc.gravity;
    for (auto& n : grid)
        if (n.mass > (R)kFltEps) n.force[1] = (R)((double)n.force[1] - g * (double)n.mass);
}

// CollocatedGridData3D::updateVelocity (src/grid3d.cu:36-41).
template <class R>
void Solver<R>::updateGridVelocities(R dt) {
    for (auto& n : grid) {
        if (n.mass > (R)kFltEps) {
            for (int a = 0; a < 3; ++a) n.velocity[a] /= n.mass;
            for (int a = 0; a < 3; ++a) n.velocity_star[a] = n.velocity[a] + dt * n.force[a] / n.mass;
        }
    }
}

// gridCollision (src/mpm_solver3d.cu:405-426), or the sticky-wall option.
template <class R>
void Solver<R>::gridCollision(R dt) {
    R fr = (R)desc.friction;
    for (int z = 0; z < res[2]; ++z)
        for (int y = 0; y < res[1]; ++y)
            for (int x = 0; x < res[0]; ++x) {
                Node<R>& n = grid[(size_t)x + (size_t)res[0] * ((size_t)y + (size_t)res[1] * z)];
                int idx[3] = {x, y, z};
                if (desc.boundary == MPM_BOUNDARY_STICKY) {
                    int t = desc.sticky_cells;
                    bool wall = false;
                    for (int a = 0; a < 3; ++a) wall |= (idx[a] < t) || (idx[a] >= res[a] - t);
                    if (wall) n.velocity_star = Vec3<R>{};
                } else {
                    Vec3<R> pos;
                    for (int a = 0; a < 3; ++a) pos[a] = (origin[a] + h * (R)idx[a]) + dt * n.velocity_star[a];
                    n.velocity_star = applyBoundaryCollision(pos, n.velocity_star, origin, target, fr);
                }
                if (has_phi) {
                    Vec3<R> pos;
                    for (int a = 0; a < 3; ++a) pos[a] = (origin[a] + h * (R)idx[a]) + dt * n.velocity_star[a];
                    n.velocity_star = applyLevelSetCollision(pos, n.velocity_star, phi.data(), res, origin, h,
                                                             phi_friction, phi_vel);
                }
            }
}

// gridToParticles (PIC-FLIP src/mpm_solver3d.cu:316-379; APIC
// src/apic_mpm_solver3d.cu:326-388).
template <class R>
void Solver<R>::gridToParticles(R dt, R blend) {
    const bool apic = desc.transfer == MPM_TRANSFER_APIC;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long i = 0; i < (long long)particles.size(); ++i) {
        Particle<R>& p = particles[i];
        Mat3<R> gradv{};
        Vec3<R> vpic{}, vflip = p.v;
        Mat3<R> B{};
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            R w = weight3D(desc.interpolation, p.x, gp, h);
            Vec3<R> g = weightGradient3D(desc.interpolation, p.x, gp, h);
            const Node<R>& n = grid[gi];
            Vec3<R> vi;
            for (int a = 0; a < 3; ++a) vi[a] = n.velocity_star[a] * w;
            for (int a = 0; a < 3; ++a) vpic[a] += vi[a];
            if (apic) {
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) B(a, b) += vi[a] * (gp[b] - p.x[b]);
            } else {
                for (int a = 0; a < 3; ++a) vflip[a] += (n.velocity_star[a] - n.velocity[a]) * w;
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) gradv(a, b) += n.velocity_star[a] * g[b];
        });
        Vec3<R> vel;
        if (apic) {
            vel = vpic;
            p.B = B;
        } else {
            R om = (R)(1.0 - (double)blend);
            for (int a = 0; a < 3; ++a) vel[a] = blend * vflip[a] + om * vpic[a];
        }
        updateDeformationGradient(p, gradv, dt);
        p.v = vel;
    }
}

template <class R>
void Solver<R>::particlesCollision(R dt) {
    R fr = (R)desc.friction;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long i = 0; i < (long long)particles.size(); ++i) {
        Particle<R>& p = particles[i];
        Vec3<R> pos;
        for (int a = 0; a < 3; ++a) pos[a] = p.x[a] + dt * p.v[a];
        p.v = applyBoundaryCollision(pos, p.v, origin, target, fr);
        if (has_phi) {
            for (int a = 0; a < 3; ++a) pos[a] = p.x[a] + dt * p.v[a];
            p.v = applyLevelSetCollision(pos, p.v, phi.data(), res, origin, h, phi_friction, phi_vel);
        }
    }
}

template <class R>
void Solver<R>::advectParticles(R dt) {
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long i = 0; i < (long long)particles.size(); ++i)
        for (int a = 0; a < 3; ++a) particles[i].x[a] += dt * particles[i].v[a];
}

// Hessian action and the semi-implicit solve (Stomakhin et al. 2013, section
// 9: sum_j (I delta_ij + beta dt^2 m_i^-1 d2Phi/dx_i dx_j) v_j = v*_i, solved
// here in the symmetric form (M + beta dt^2 H) v = M v* by conjugate
// residual).  Unknowns are the nodes with m > FLT_EPSILON (the velocity
// update's threshold, src/grid3d.cu:36-41).
template <class R>
void Solver<R>::hessianAction(const std::vector<Vec3<R>>& u, std::vector<Vec3<R>>& out) {
    std::vector<Mat3<R>> T(particles.size());
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long i = 0; i < (long long)particles.size(); ++i) {
        const Particle<R>& p = particles[i];
        Mat3<R> G{};
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            Vec3<R> g = weightGradient3D(desc.interpolation, p.x, gp, h);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) G(a, b) += u[gi][a] * g[b];
        });
        Mat3<R> dP = stressDifferential(p, matmul(G, p.Fe));
        Mat3<R> t = matmul(dP, transpose(p.Fe));
        for (int k = 0; k < 9; ++k) t.a[k] *= p.volume0;
        T[i] = t;
    }
    out.assign(grid.size(), Vec3<R>{});
    scatterDeterministic([&](size_t i) {
        const Particle<R>& p = particles[i];
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            Vec3<R> g = weightGradient3D(desc.interpolation, p.x, gp, h);
            for (int a = 0; a < 3; ++a) out[gi][a] += T[i](a, 0) * g[0] + T[i](a, 1) * g[1] + T[i](a, 2) * g[2];
        });
    });
}

template <class R>
void Solver<R>::displacedForce(const std::vector<Vec3<R>>& d, std::vector<Vec3<R>>& out) {
    std::vector<Mat3<R>> T(particles.size());
    for (size_t i = 0; i < particles.size(); ++i) {
        Particle<R> p = particles[i];
        Mat3<R> G{};
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            Vec3<R> g = weightGradient3D(desc.interpolation, p.x, gp, h);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) G(a, b) += d[gi][a] * g[b];
        });
        const Mat3<R> F0 = p.Fe;
        Mat3<R> A = Mat3<R>::identity();
        for (int k = 0; k < 9; ++k) A.a[k] += G.a[k];
        p.Fe = matmul(A, F0);
        // tau = V0 P(F^) F^^T, so V0 P(F^) F0^T = tau F^^-T F0^T
        const Mat3<R> tau = volumeTimesCauchyStress(p);
        const Mat3<R> C = cofactor(p.Fe);
        const R J = det3(p.Fe);
        Mat3<R> FiT{};
        for (int k = 0; k < 9; ++k) FiT.a[k] = C.a[k] / J;
        T[i] = matmul(matmul(tau, FiT), transpose(F0));
    }
    out.assign(grid.size(), Vec3<R>{});
    for (size_t i = 0; i < particles.size(); ++i) {
        const Particle<R>& p = particles[i];
        forEachNode(p, [&](size_t gi, const Vec3<R>& gp) {
            Vec3<R> g = weightGradient3D(desc.interpolation, p.x, gp, h);
            for (int a = 0; a < 3; ++a) out[gi][a] -= T[i](a, 0) * g[0] + T[i](a, 1) * g[1] + T[i](a, 2) * g[2];
        });
    }
}

template <class R>
void Solver<R>::solveLinearSystem(R dt) {
    last_iters = 0;
    last_residual = 0;
    if (!(beta > 0)) return;
    // Conjugate residual preconditioned by the node masses (z = M^-1 r): the
    // masses span orders of magnitude between the interior and the edge of a
    // body, and the unpreconditioned iteration stalls on the light nodes.
    const size_t nn = grid.size();
    const R c = beta * dt * dt;
    std::vector<char> act(nn);
    std::vector<R> m(nn);
    std::vector<Vec3<R>> x(nn), r(nn), z(nn), pv(nn), Az(nn), Ap(nn), hv;
    for (size_t i = 0; i < nn; ++i) {
        act[i] = grid[i].mass > (R)kFltEps;
        m[i] = act[i] ? grid[i].mass : (R)0;
        x[i] = act[i] ? grid[i].velocity_star : Vec3<R>{};
    }
    auto dot = [&](const std::vector<Vec3<R>>& a, const std::vector<Vec3<R>>& b) {
        R s = 0;
        for (size_t i = 0; i < nn; ++i)
            if (act[i]) s += a[i][0] * b[i][0] + a[i][1] * b[i][1] + a[i][2] * b[i][2];
        return s;
    };
    R bb = 0;
    for (size_t i = 0; i < nn; ++i)
        for (int a = 0; a < 3; ++a) bb += (m[i] * x[i][a]) * (m[i] * x[i][a]);
    // x0 = v*: r0 = M v* - (M x0 + c H x0) = -c H v*
    hessianAction(x, hv);
    for (size_t i = 0; i < nn; ++i)
        for (int a = 0; a < 3; ++a) {
            r[i][a] = act[i] ? -c * hv[i][a] : (R)0;
            z[i][a] = act[i] ? r[i][a] / m[i] : (R)0;
        }
    R rr = dot(r, r);
    hessianAction(z, hv);
    for (size_t i = 0; i < nn; ++i)
        for (int a = 0; a < 3; ++a) {
            Az[i][a] = act[i] ? m[i] * z[i][a] + c * hv[i][a] : (R)0;
            pv[i][a] = z[i][a];
            Ap[i][a] = Az[i][a];
        }
    R zAz = dot(z, Az);
    auto apq = [&]() {  // (Ap, M^-1 Ap)
        R s = 0;
        for (size_t i = 0; i < nn; ++i)
            if (act[i]) s += (Ap[i][0] * Ap[i][0] + Ap[i][1] * Ap[i][1] + Ap[i][2] * Ap[i][2]) / m[i];
        return s;
    };
    R Apq = apq();
    int k = 0;
    for (; k < max_iter; ++k) {
        if (rr <= tol * tol * bb || !(Apq > 0)) break;
        const R alpha = zAz / Apq;
        for (size_t i = 0; i < nn; ++i)
            if (act[i])
                for (int a = 0; a < 3; ++a) {
                    x[i][a] += alpha * pv[i][a];
                    r[i][a] -= alpha * Ap[i][a];
                    z[i][a] -= alpha * (Ap[i][a] / m[i]);
                }
        rr = dot(r, r);
        hessianAction(z, hv);
        for (size_t i = 0; i < nn; ++i)
            for (int a = 0; a < 3; ++a) Az[i][a] = act[i] ? m[i] * z[i][a] + c * hv[i][a] : (R)0;
        const R zAz1 = dot(z, Az);
        const R gam = zAz1 / zAz;
        zAz = zAz1;
        for (size_t i = 0; i < nn; ++i)
            for (int a = 0; a < 3; ++a) {
                pv[i][a] = z[i][a] + gam * pv[i][a];
                Ap[i][a] = Az[i][a] + gam * Ap[i][a];
            }
        Apq = apq();
    }
    for (size_t i = 0; i < nn; ++i)
        if (act[i]) grid[i].velocity_star = x[i];
    last_iters = k;
    last_residual = bb > 0 ? std::sqrt((double)rr / (double)bb) : 0.0;
}

template <class R>
void Solver<R>::simulateOneStep() {
    R dt = (R)desc.dt;
    if (cfl > 0) {  // CFL step from the velocities the step starts with
        R m = 0;
        for (const Particle<R>& p : particles) m = std::max(m, (p.v[0] * p.v[0] + p.v[1] * p.v[1]) + p.v[2] * p.v[2]);
        const R vmax = std::sqrt(m);
        if (vmax > 0) dt = std::min(dt, (cfl * h) / vmax);
    }
    last_dt = dt;
    time += (double)dt;
    resetGrid();
    particlesToGrid();
    computeGravityForces();
    updateGridVelocities(dt);
    gridCollision(dt);
    if (beta > 0) {  // semi-implicit: solve, then the boundary again on the solved velocities
        solveLinearSystem(dt);
        gridCollision(dt);
    }
    gridToParticles(dt, (R)desc.blend);
    if (enable_particles_collision) particlesCollision(dt);
    advectParticles(dt);
}

template class Solver<float>;
template class Solver<double>;

}  // namespace oracle

// ---------------------------------------------------------------------------
// C ABI for ctypes (tests and bench only).
// ---------------------------------------------------------------------------
using namespace oracle;

namespace {
struct Handle {
    int bits;
    Solver<float>* f = nullptr;
    Solver<double>* d = nullptr;
};
thread_local std::string g_err;
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_solver_create(int bits, const mpm_scene_desc* d, const mpm_particles_in* in) {
    try {
        Handle* h = new Handle;
        h->bits = bits;
        if (bits == 32)
            h->f = new Solver<float>(*d, *in);
        else
            h->d = new Solver<double>(*d, *in);
        return h;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_solver_destroy(void* p) {
    Handle* h = (Handle*)p;
    delete h->f;
    delete h->d;
    delete h;
}

#define DISPATCH(h, call)        \
    do {                         \
        if ((h)->f)              \
            (h)->f->call;        \
        else                     \
            (h)->d->call;        \
    } while (0)

void orc_set_threads(void* p, int t) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->threads = t;
    if (h->d) h->d->threads = t;
}
void orc_set_particles_collision(void* p, int e) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->enable_particles_collision = e != 0;
    if (h->d) h->d->enable_particles_collision = e != 0;
}
void orc_initialize(void* p) { DISPATCH((Handle*)p, initialize()); }
void orc_reset_grid(void* p) { DISPATCH((Handle*)p, resetGrid()); }
void orc_particles_to_grid(void* p) { DISPATCH((Handle*)p, particlesToGrid()); }
void orc_gravity(void* p) { DISPATCH((Handle*)p, computeGravityForces()); }
void orc_update_grid_velocities(void* p, double dt) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->updateGridVelocities((float)dt);
    else h->d->updateGridVelocities(dt);
}
void orc_grid_collision(void* p, double dt) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->gridCollision((float)dt);
    else h->d->gridCollision(dt);
}
void orc_grid_to_particles(void* p, double dt, double blend) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->gridToParticles((float)dt, (float)blend);
    else h->d->gridToParticles(dt, blend);
}
void orc_particles_collision(void* p, double dt) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->particlesCollision((float)dt);
    else h->d->particlesCollision(dt);
}
void orc_advect(void* p, double dt) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->advectParticles((float)dt);
    else h->d->advectParticles(dt);
}
void orc_step(void* p, int n) {
    for (int i = 0; i < n; ++i) DISPATCH((Handle*)p, simulateOneStep());
}

// Particle field export as double (fields as in MPM_FIELD_*).
int orc_get_particles(void* p, int field, double* out) {
    Handle* h = (Handle*)p;
    auto fill = [&](auto* s) {
        size_t n = s->particles.size();
        for (size_t i = 0; i < n; ++i) {
            auto& q = s->particles[i];
            switch (field) {
                case MPM_FIELD_POSITION: for (int a = 0; a < 3; ++a) out[3 * i + a] = q.x[a]; break;
                case MPM_FIELD_VELOCITY: for (int a = 0; a < 3; ++a) out[3 * i + a] = q.v[a]; break;
                case MPM_FIELD_FE: for (int a = 0; a < 9; ++a) out[9 * i + a] = q.Fe.a[a]; break;
                case MPM_FIELD_FP: for (int a = 0; a < 9; ++a) out[9 * i + a] = q.Fp.a[a]; break;
                case MPM_FIELD_B: for (int a = 0; a < 9; ++a) out[9 * i + a] = q.B.a[a]; break;
                case MPM_FIELD_VOLUME0: out[i] = q.volume0; break;
                case MPM_FIELD_MASS: out[i] = q.mass; break;
                case MPM_FIELD_DET_FE: out[i] = det3(q.Fe); break;
                case MPM_FIELD_DET_FP: out[i] = det3(q.Fp); break;
                default: return 1;
            }
        }
        return 0;
    };
    return h->f ? fill(h->f) : fill(h->d);
}

int orc_set_particles(void* p, int field, const double* in) {
    Handle* h = (Handle*)p;
    auto put = [&](auto* s) {
        using RR = std::remove_reference_t<decltype(s->particles[0].mass)>;
        size_t n = s->particles.size();
        for (size_t i = 0; i < n; ++i) {
            auto& q = s->particles[i];
            switch (field) {
                case MPM_FIELD_POSITION: for (int a = 0; a < 3; ++a) q.x[a] = (RR)in[3 * i + a]; break;
                case MPM_FIELD_VELOCITY: for (int a = 0; a < 3; ++a) q.v[a] = (RR)in[3 * i + a]; break;
                case MPM_FIELD_FE: for (int a = 0; a < 9; ++a) q.Fe.a[a] = (RR)in[9 * i + a]; break;
                case MPM_FIELD_FP: for (int a = 0; a < 9; ++a) q.Fp.a[a] = (RR)in[9 * i + a]; break;
                case MPM_FIELD_B: for (int a = 0; a < 9; ++a) q.B.a[a] = (RR)in[9 * i + a]; break;
                case MPM_FIELD_VOLUME0: q.volume0 = (RR)in[i]; break;
                default: return 1;
            }
        }
        return 0;
    };
    return h->f ? put(h->f) : put(h->d);
}

int orc_get_grid(void* p, int field, double* out) {
    Handle* h = (Handle*)p;
    auto fill = [&](auto* s) {
        size_t n = s->grid.size();
        for (size_t i = 0; i < n; ++i) {
            auto& g = s->grid[i];
            switch (field) {
                case MPM_GRID_MASS: out[i] = g.mass; break;
                case MPM_GRID_VELOCITY: for (int a = 0; a < 3; ++a) out[3 * i + a] = g.velocity[a]; break;
                case MPM_GRID_FORCE: for (int a = 0; a < 3; ++a) out[3 * i + a] = g.force[a]; break;
                case MPM_GRID_VELOCITY_STAR: for (int a = 0; a < 3; ++a) out[3 * i + a] = g.velocity_star[a]; break;
                default: return 1;
            }
        }
        return 0;
    };
    return h->f ? fill(h->f) : fill(h->d);
}

// --- Known-answer helpers ---------------------------------------------------
void orc_spline(int bits, int type, const double* x, int n, double* N, double* dN) {
    for (int i = 0; i < n; ++i) {
        if (bits == 32) {
            N[i] = splineN<float>(type, (float)x[i]);
            dN[i] = splineNDot<float>(type, (float)x[i]);
        } else {
            N[i] = splineN<double>(type, x[i]);
            dN[i] = splineNDot<double>(type, x[i]);
        }
    }
}

// mode: 0 = McAdams float (4 sweeps), 1 = McAdams double (4 sweeps), 2 = exact double.
void orc_svd3(int mode, const double* A, double* U, double* s, double* V) {
    if (mode == 0) {
        Mat3<float> a, u, v;
        Vec3<float> ss;
        for (int i = 0; i < 9; ++i) a.a[i] = (float)A[i];
        svdMcAdams<float>(a, u, ss, v, 4);
        for (int i = 0; i < 9; ++i) {
            U[i] = u.a[i];
            V[i] = v.a[i];
        }
        for (int i = 0; i < 3; ++i) s[i] = ss[i];
    } else {
        Mat3<double> a, u, v;
        Vec3<double> ss;
        for (int i = 0; i < 9; ++i) a.a[i] = A[i];
        if (mode == 1)
            svdMcAdams<double>(a, u, ss, v, 4);
        else
            svdExact(a, u, ss, v);
        for (int i = 0; i < 9; ++i) {
            U[i] = u.a[i];
            V[i] = v.a[i];
        }
        for (int i = 0; i < 3; ++i) s[i] = ss[i];
    }
}

void orc_collision(int bits, const double* pos, const double* vel, const double* lo, const double* hi,
                   double friction, double* out) {
    if (bits == 32) {
        Vec3<float> p, v, a, b;
        for (int i = 0; i < 3; ++i) {
            p[i] = (float)pos[i];
            v[i] = (float)vel[i];
            a[i] = (float)lo[i];
            b[i] = (float)hi[i];
        }
        Vec3<float> r = applyBoundaryCollision<float>(p, v, a, b, (float)friction);
        for (int i = 0; i < 3; ++i) out[i] = r[i];
    } else {
        Vec3<double> p, v, a, b;
        for (int i = 0; i < 3; ++i) {
            p[i] = pos[i];
            v[i] = vel[i];
            a[i] = lo[i];
            b[i] = hi[i];
        }
        Vec3<double> r = applyBoundaryCollision<double>(p, v, a, b, friction);
        for (int i = 0; i < 3; ++i) out[i] = r[i];
    }
}

void orc_set_implicit(void* p, double beta, int max_iter, double tol) {
    Handle* h = (Handle*)p;
    auto set = [&](auto* s) {
        using RR = typename std::remove_pointer<decltype(s)>::type::Real;
        s->beta = (RR)beta;
        s->max_iter = max_iter;
        s->tol = (RR)tol;
    };
    if (h->f) set(h->f);
    else set(h->d);
}
void orc_solve_linear_system(void* p, double dt) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->solveLinearSystem((float)dt);
    else h->d->solveLinearSystem(dt);
}
void orc_solve_info(void* p, int* iters, double* residual) {
    Handle* h = (Handle*)p;
    *iters = h->f ? h->f->last_iters : h->d->last_iters;
    *residual = h->f ? h->f->last_residual : h->d->last_residual;
}
// which = 0: hessianAction(u), 1: displacedForce(u); u and out: nodes x 3
void orc_grid_operator(void* p, int which, const double* u, double* out) {
    Handle* h = (Handle*)p;
    auto run = [&](auto* s) {
        using RR = typename std::remove_pointer<decltype(s)>::type::Real;
        const size_t nn = s->grid.size();
        std::vector<Vec3<RR>> in(nn), res;
        for (size_t i = 0; i < nn; ++i)
            for (int a = 0; a < 3; ++a) in[i][a] = (RR)u[3 * i + a];
        if (which == 0) s->hessianAction(in, res);
        else s->displacedForce(in, res);
        for (size_t i = 0; i < nn; ++i)
            for (int a = 0; a < 3; ++a) out[3 * i + a] = (double)res[i][a];
    };
    if (h->f) run(h->f);
    else run(h->d);
}

void orc_set_cfl(void* p, double cfl) {
    Handle* h = (Handle*)p;
    if (h->f) h->f->cfl = (float)cfl;
    else h->d->cfl = cfl;
}
void orc_time(void* p, double* t, double* last_dt) {
    Handle* h = (Handle*)p;
    *t = h->f ? h->f->time : h->d->time;
    *last_dt = h->f ? (double)h->f->last_dt : h->d->last_dt;
}

int orc_set_level_set(void* p, const double* phi, double friction, const double* vel) {
    Handle* h = (Handle*)p;
    auto set = [&](auto* s) {
        using RR = typename std::remove_pointer<decltype(s)>::type::Real;
        s->has_phi = phi != nullptr;
        s->phi.clear();
        if (!phi) return;
        const size_t nodes = (size_t)s->res[0] * s->res[1] * s->res[2];
        s->phi.resize(nodes);
        for (size_t i = 0; i < nodes; ++i) s->phi[i] = (RR)phi[i];
        s->phi_friction = (RR)friction;
        for (int a = 0; a < 3; ++a) s->phi_vel[a] = vel ? (RR)vel[a] : (RR)0;
    };
    for (int a = 0; a < 3; ++a)
        if (phi && (h->f ? h->f->res[a] : h->d->res[a]) < 2) {
            g_err = "a level set needs >= 2 nodes per axis";
            return 1;
        }
    if (h->f) set(h->f);
    else set(h->d);
    return 0;
}

// One level-set collision (known-answer tests).
void orc_level_set_collision(int bits, const int* res, const double* origin, double h, const double* phi,
                             double friction, const double* vco, const double* pos, const double* vel, double* out) {
    auto run = [&](auto tag) {
        using RR = decltype(tag);
        const size_t nodes = (size_t)res[0] * res[1] * res[2];
        std::vector<RR> ph(nodes);
        for (size_t i = 0; i < nodes; ++i) ph[i] = (RR)phi[i];
        Vec3<RR> o, vc, p, v;
        for (int a = 0; a < 3; ++a) {
            o[a] = (RR)origin[a];
            vc[a] = (RR)vco[a];
            p[a] = (RR)pos[a];
            v[a] = (RR)vel[a];
        }
        Vec3<RR> r = applyLevelSetCollision<RR>(p, v, ph.data(), res, o, (RR)h, (RR)friction, vc);
        for (int a = 0; a < 3; ++a) out[a] = (double)r[a];
    };
    if (bits == 32) run(0.0f);
    else run(0.0);
}

// Stress of one particle state (V0 * P F^T as volumeTimesCauchyStress returns).
void orc_stress(int bits, int model, const double* Fe, const double* Fp, double mu0, double la0, double xi,
                double V0, double* out, double* Fe_out) {
    auto run = [&](auto tag) {
        using RR = decltype(tag);
        Particle<RR> p{};
        for (int i = 0; i < 9; ++i) {
            p.Fe.a[i] = (RR)Fe[i];
            p.Fp.a[i] = (RR)Fp[i];
        }
        p.mu0 = (RR)mu0;
        p.lambda0 = (RR)la0;
        p.xi = (RR)xi;
        p.volume0 = (RR)V0;
        p.model = model;
        Mat3<RR> s = volumeTimesCauchyStress(p);
        for (int i = 0; i < 9; ++i) {
            out[i] = s.a[i];
            Fe_out[i] = p.Fe.a[i];
        }
    };
    if (bits == 32) run(float{});
    else run(double{});
}

// One plasticity update of a particle (Fe, Fp in/out).
void orc_update_deformation(int bits, double* Fe, double* Fp, const double* gradv, double dt, double tc, double ts) {
    auto run = [&](auto tag) {
        using RR = decltype(tag);
        Particle<RR> p{};
        Mat3<RR> g;
        for (int i = 0; i < 9; ++i) {
            p.Fe.a[i] = (RR)Fe[i];
            p.Fp.a[i] = (RR)Fp[i];
            g.a[i] = (RR)gradv[i];
        }
        p.theta_c = (RR)tc;
        p.theta_s = (RR)ts;
        updateDeformationGradient(p, g, (RR)dt);
        for (int i = 0; i < 9; ++i) {
            Fe[i] = p.Fe.a[i];
            Fp[i] = p.Fp.a[i];
        }
    };
    if (bits == 32) run(float{});
    else run(double{});
}

}  // extern "C"
