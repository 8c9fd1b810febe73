// chains/mpm_b200.hpp -- header-only C++ facade with the reference's API.
//
// Mirrors namespace chains of H-YWu/mpm: InterpolationType and
// ConstitutiveModel (include/enums.h), MaterialPoint3D's constructor
// (include/material_point3d.h:26-37), MPMSolver3D / APICMPMSolver3D
// (include/mpm_solver3d.h:21-96, include/apic_mpm_solver3d.h:20-92),
// MPM3DConfiguration / parseYAML (include/mpm3d_parser.h:13-37) and the
// builders (include/mpm_solver3d_builder.h:10-12), on top of the C ABI.
// Eigen vectors become Vec3f / Vec3i; thrust::host_vector becomes
// std::vector; GL and OpenVDB outputs become downloads.  Errors throw
// std::runtime_error with the library's message.  Solvers are move-only (the
// reference's copy was an unguarded shallow copy).
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../mpm_b200.h"
#include "../mpm_b200_config.h"

namespace chains {

enum class InterpolationType { LINEAR = 0, QUADRATIC_BSPLINE = 1, CUBIC_BSPLINE = 2 };
enum class ConstitutiveModel { FIXED_COROTATED = 0, NEO_HOOKEAN = 1 };
enum class IntegrationType { EXPLICIT, SEMI_IMPLICIT, FULL_IMPLICIT };

struct Vec3f {
    float x = 0.f, y = 0.f, z = 0.f;
};
struct Vec3i {
    int x = 0, y = 0, z = 0;
};

inline void check(mpm_status st, const char* where) {
    if (st != MPM_OK) throw std::runtime_error(std::string(where) + ": " + mpm_last_error_string());
}

// Host-side particle as the reference constructs it (src/material_point3d.cu:10-30).
struct MaterialPoint3D {
    Vec3f position, velocity;
    float mass = 0.f;
    float hardening_coefficient = 0.f, youngs_modulus = 0.f, poisson_ratio = 0.f;
    float critical_compression = 0.f, critical_stretch = 0.f;
    ConstitutiveModel constitutive_model = ConstitutiveModel::FIXED_COROTATED;

    MaterialPoint3D() = default;
    MaterialPoint3D(Vec3f particlePosition, Vec3f particleVelocity, float particleMass, float hardeningCoefficient,
                    float YoungModulus, float PoissonRatio, float criticalCompression, float criticleStretch,
                    ConstitutiveModel constitutiveModel)
        : position(particlePosition), velocity(particleVelocity), mass(particleMass),
          hardening_coefficient(hardeningCoefficient), youngs_modulus(YoungModulus), poisson_ratio(PoissonRatio),
          critical_compression(criticalCompression), critical_stretch(criticleStretch),
          constitutive_model(constitutiveModel) {}
};
using APICMaterialPoint3D = MaterialPoint3D;

// LevelSetCollisionObject3D (include/collision_object3d.h:9-12): signed
// distance per grid node (index x + X (y + Y z), negative inside), here in
// float with the object's friction and surface velocity.
struct LevelSetCollisionObject3D {
    std::vector<float> level_set;
    float friction = 0.f;
    Vec3f velocity;
};

namespace detail {

class SolverBase {
public:
    bool enableParticlesCollision() const {
        int32_t e = 0;
        check(mpm_solver_get_particles_collision(h_, &e), "_enable_particles_collision");
        return e != 0;
    }
    void switchIfEnableParticlesCollision() {
        check(mpm_solver_set_particles_collision(h_, enableParticlesCollision() ? 0 : 1),
              "switchIfEnableParticlesCollision");
    }
    void simulateOneStep() { check(mpm_solver_step(h_, 1), "simulateOneStep"); }
    void step(int n) { check(mpm_solver_step(h_, n), "step"); }
    void synchronize() { check(mpm_solver_synchronize(h_), "synchronize"); }
    void initialize() { check(mpm_solver_initialize(h_), "initialize"); }
    void resetGrid() { check(mpm_solver_reset_grid(h_), "resetGrid"); }
    void particlesToGrid() { check(mpm_solver_particles_to_grid(h_), "particlesToGrid"); }
    void computeExternalForces() { check(mpm_solver_compute_external_forces(h_), "computeExternalForces"); }
    void computeGravityForces() { check(mpm_solver_compute_gravity_forces(h_), "computeGravityForces"); }
    void updateGridVelocities(float dt) { check(mpm_solver_update_grid_velocities(h_, dt), "updateGridVelocities"); }
    void solveLinearSystem(float dt) { check(mpm_solver_solve_linear_system(h_, dt), "solveLinearSystem"); }
    void gridCollision(float dt) { check(mpm_solver_grid_collision(h_, dt), "gridCollision"); }
    void particlesCollision(float dt) { check(mpm_solver_particles_collision(h_, dt), "particlesCollision"); }
    void advectParticles(float dt) { check(mpm_solver_advect_particles(h_, dt), "advectParticles"); }

    size_t numParticles() const {
        size_t n = 0;
        check(mpm_solver_num_particles(h_, &n), "numParticles");
        return n;
    }
    // Headless replacement of updateGLBufferWithCUDA()/updateGLBufferByCPU():
    // (x, y, z, 1) per particle in the construction order.
    std::vector<float> positions4() {
        std::vector<float> out(4 * numParticles());
        check(mpm_solver_download(h_, MPM_FIELD_POSITION4, out.data()), "positions4");
        return out;
    }
    // Density grid sum_p m_p w_ip / h^3 (what writeToOpenVDB rasterises),
    // res.x * res.y * res.z floats, index x + X (y + Y z).
    std::vector<float> density() {
        mpm_scene_desc d{};
        check(mpm_solver_get_desc(h_, &d), "density");
        std::vector<float> out((size_t)d.resolution[0] * d.resolution[1] * d.resolution[2]);
        check(mpm_solver_download_density(h_, out.data()), "density");
        return out;
    }
    // writeToOpenVDB (include/mpm_solver3d.h:74): the density grid as an
    // OpenVDB file with one FloatGrid named "density" (mpm_solver_write_vdb).
    void writeToOpenVDB(std::string filePath) { check(mpm_solver_write_vdb(h_, filePath.c_str()), "writeToOpenVDB"); }
    // Launch settings and the autotuner (mpm_solver_autotune); results are
    // bitwise the same for any setting.
    mpm_tuning autotune(int stepsPerCandidate = 3, int flags = 0) {
        check(mpm_solver_autotune(h_, stepsPerCandidate, flags, nullptr), "autotune");
        mpm_tuning t{};
        check(mpm_solver_get_tuning(h_, &t), "autotune");
        return t;
    }
    // Applies the object in every grid collision (mpm_solver_set_level_set).
    void setCollisionObject(const LevelSetCollisionObject3D& obj) {
        const float v[3] = {obj.velocity.x, obj.velocity.y, obj.velocity.z};
        mpm_scene_desc d{};
        check(mpm_solver_get_desc(h_, &d), "setCollisionObject");
        if (obj.level_set.size() != (size_t)d.resolution[0] * d.resolution[1] * d.resolution[2])
            throw std::runtime_error("setCollisionObject: level set size does not match the grid");
        check(mpm_solver_set_level_set(h_, obj.level_set.data(), obj.friction, v), "setCollisionObject");
    }
    // IntegrationType (include/enums.h:17-21): EXPLICIT, SEMI_IMPLICIT (beta
    // 1/2) or FULL_IMPLICIT (backward Euler, beta 1), see mpm_solver_set_implicit.
    void setIntegrationType(IntegrationType t, int maxIterations = 50, float tolerance = 1e-5f) {
        const float beta = t == IntegrationType::EXPLICIT ? 0.f : (t == IntegrationType::SEMI_IMPLICIT ? 0.5f : 1.f);
        check(mpm_solver_set_implicit(h_, beta, maxIterations, tolerance), "setIntegrationType");
    }
    // CFL time step (mpm_solver_set_cfl) and the simulated time.
    void setCfl(float cfl) { check(mpm_solver_set_cfl(h_, cfl), "setCfl"); }
    double simulatedTime() {
        double t = 0.0;
        check(mpm_solver_time(h_, &t, nullptr), "simulatedTime");
        return t;
    }
    void clearCollisionObject() { check(mpm_solver_set_level_set(h_, nullptr, 0.f, nullptr), "clearCollisionObject"); }
    std::vector<float> download(int field, int comps) {
        std::vector<float> out((size_t)comps * numParticles());
        check(mpm_solver_download(h_, field, out.data()), "download");
        return out;
    }
    mpm_solver* handle() { return h_; }
    // Checkpoint of the full state (mpm_solver_save); resume with the
    // solver class's fromCheckpoint().
    void save(const std::string& path) { check(mpm_solver_save(h_, path.c_str()), "save"); }

    SolverBase(const SolverBase&) = delete;
    SolverBase& operator=(const SolverBase&) = delete;
    SolverBase(SolverBase&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    SolverBase& operator=(SolverBase&& o) noexcept {
        if (this != &o) {
            if (h_) mpm_solver_destroy(h_);
            h_ = o.h_;
            o.h_ = nullptr;
        }
        return *this;
    }
    ~SolverBase() {
        if (h_) mpm_solver_destroy(h_);
    }

protected:
    SolverBase() = default;
    explicit SolverBase(mpm_solver* h) : h_(h) {}

    void create(const std::vector<MaterialPoint3D>& particles, Vec3f origin, Vec3i res, float stride, float friction,
                float blend, InterpolationType interp, float dt, int transfer) {
        // one material per distinct constant tuple, a material id per particle
        std::vector<float> x, v, m;
        std::vector<uint16_t> ids;
        std::vector<mpm_material> mats;
        std::map<std::tuple<float, float, float, float, float, int>, uint16_t> index;
        for (const auto& p : particles) {
            auto key = std::make_tuple(p.youngs_modulus, p.poisson_ratio, p.hardening_coefficient,
                                       p.critical_compression, p.critical_stretch, (int)p.constitutive_model);
            auto it = index.find(key);
            if (it == index.end()) {
                if (mats.size() >= 65535) throw std::runtime_error("too many distinct materials");
                it = index.emplace(key, (uint16_t)mats.size()).first;
                mats.push_back({p.youngs_modulus, p.poisson_ratio, p.hardening_coefficient, p.critical_compression,
                                p.critical_stretch, (int32_t)p.constitutive_model});
            }
            ids.push_back(it->second);
            x.insert(x.end(), {p.position.x, p.position.y, p.position.z});
            v.insert(v.end(), {p.velocity.x, p.velocity.y, p.velocity.z});
            m.push_back(p.mass);
        }
        if (mats.empty()) mats.push_back({1.4e5f, 0.2f, 10.f, 2.5e-2f, 7.5e-3f, MPM_MODEL_FIXED_COROTATED});
        mpm_scene_desc d{};
        d.origin[0] = origin.x;
        d.origin[1] = origin.y;
        d.origin[2] = origin.z;
        d.resolution[0] = res.x;
        d.resolution[1] = res.y;
        d.resolution[2] = res.z;
        d.stride = stride;
        d.friction = friction;
        d.blend = blend;
        d.dt = dt;
        d.gravity = 9.80665f;  // hard-coded in the reference (src/mpm_solver3d.cu:397)
        d.transfer = transfer;
        d.interpolation = (int32_t)interp;
        d.boundary = MPM_BOUNDARY_REFERENCE;
        d.sticky_cells = 3;
        d.volume_mode = MPM_VOLUME_GRID_ESTIMATE;
        d.particles_collision = 0;
        mpm_particles_in in{};
        in.n = m.size();
        in.position = x.data();
        in.velocity = v.data();
        in.mass = m.data();
        in.material = mats.size() > 1 ? ids.data() : nullptr;
        in.materials = mats.data();
        in.nmaterials = (int32_t)mats.size();
        check(mpm_solver_create(&d, &in, &h_), "MPMSolver3D");
    }

    mpm_solver* h_ = nullptr;
};

}  // namespace detail

// PIC-FLIP solver (include/mpm_solver3d.h:25-34).
class MPMSolver3D : public detail::SolverBase {
public:
    MPMSolver3D(const std::vector<MaterialPoint3D>& particles, Vec3f gridOrigin, Vec3i gridResolution,
                float gridStride, float gridBoundaryFrictionCoefficient, float blendCoefficient,
                InterpolationType interpolationType, float deltaTime) {
        create(particles, gridOrigin, gridResolution, gridStride, gridBoundaryFrictionCoefficient, blendCoefficient,
               interpolationType, deltaTime, MPM_TRANSFER_PIC_FLIP);
    }
    explicit MPMSolver3D(mpm_solver* h) : SolverBase(h) {}
    static MPMSolver3D fromCheckpoint(const std::string& path) {
        mpm_solver* h = nullptr;
        check(mpm_solver_load(path.c_str(), &h), "fromCheckpoint");
        return MPMSolver3D(h);
    }
    void gridToParticles(float dt, float blendCoefficient) {
        check(mpm_solver_grid_to_particles(h_, dt, blendCoefficient), "gridToParticles");
    }
};

// APIC solver (include/apic_mpm_solver3d.h:24-32).
class APICMPMSolver3D : public detail::SolverBase {
public:
    APICMPMSolver3D(const std::vector<APICMaterialPoint3D>& particles, Vec3f gridOrigin, Vec3i gridResolution,
                    float gridStride, float gridBoundaryFrictionCoefficient, InterpolationType interpolationType,
                    float deltaTime) {
        create(particles, gridOrigin, gridResolution, gridStride, gridBoundaryFrictionCoefficient, 0.f,
               interpolationType, deltaTime, MPM_TRANSFER_APIC);
    }
    explicit APICMPMSolver3D(mpm_solver* h) : SolverBase(h) {}
    static APICMPMSolver3D fromCheckpoint(const std::string& path) {
        mpm_solver* h = nullptr;
        check(mpm_solver_load(path.c_str(), &h), "fromCheckpoint");
        return APICMPMSolver3D(h);
    }
    void gridToParticles(float dt) { check(mpm_solver_grid_to_particles(h_, dt, 0.f), "gridToParticles"); }
};

// MPM3DConfiguration (include/mpm3d_parser.h:13-33), owning the parsed C config.
class MPM3DConfiguration {
public:
    MPM3DConfiguration() = default;
    explicit MPM3DConfiguration(mpm_config* c) : c_(c) {}
    MPM3DConfiguration(const MPM3DConfiguration&) = delete;
    MPM3DConfiguration& operator=(const MPM3DConfiguration&) = delete;
    MPM3DConfiguration(MPM3DConfiguration&& o) noexcept : c_(o.c_) { o.c_ = nullptr; }
    MPM3DConfiguration& operator=(MPM3DConfiguration&& o) noexcept {
        std::swap(c_, o.c_);
        return *this;
    }
    ~MPM3DConfiguration() { mpm_config_free(c_); }
    const mpm_config& raw() const { return *c_; }
    int groups() const { return c_->ngroups; }
    std::string groupPath(int i) const { return c_->groups[i].file; }
    Vec3i resolution() const { return {c_->resolution[0], c_->resolution[1], c_->resolution[2]}; }
    float stride() const { return c_->stride; }
    float deltaTime() const { return c_->dt; }
    InterpolationType interpolation() const { return (InterpolationType)c_->interpolation; }

private:
    mpm_config* c_ = nullptr;
};

// parseYAML (src/mpm3d_parser.cpp:20-71)
inline MPM3DConfiguration parseYAML(const std::string& filePath) {
    mpm_config* c = nullptr;
    check(mpm_config_parse_yaml(filePath.c_str(), &c), "parseYAML");
    return MPM3DConfiguration(c);
}

// buildMPMSolver3DFromYAML / buildAPICMPMSolver3DFromYAML (src/mpm_solver3d_builder.cu:32-129)
inline MPMSolver3D buildMPMSolver3DFromYAML(const MPM3DConfiguration& config, int& particlesNumber) {
    mpm_solver* h = nullptr;
    int32_t n = 0;
    check(mpm_solver_create_from_config(&config.raw(), MPM_TRANSFER_PIC_FLIP, &h, &n), "buildMPMSolver3DFromYAML");
    particlesNumber = n;
    return MPMSolver3D(h);
}

inline APICMPMSolver3D buildAPICMPMSolver3DFromYAML(const MPM3DConfiguration& config, int& particlesNumber) {
    mpm_solver* h = nullptr;
    int32_t n = 0;
    check(mpm_solver_create_from_config(&config.raw(), MPM_TRANSFER_APIC, &h, &n), "buildAPICMPMSolver3DFromYAML");
    particlesNumber = n;
    return APICMPMSolver3D(h);
}

}  // namespace chains
