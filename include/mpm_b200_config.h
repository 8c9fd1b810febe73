/*
 * mpm_b200_config.h -- scene configuration (YAML) and the solver builder.
 *
 * Replaces the reference's parseYAML (include/mpm3d_parser.h:13-37,
 * src/mpm3d_parser.cpp:20-71), readXYZFile and the two builders
 * (include/mpm_solver3d_builder.h:10-12, src/mpm_solver3d_builder.cu:10-129).
 * Same YAML schema (ParticleGroups[], Grid, Transfer, Interpolation,
 * Simulate, Render) and the same .xyz semantics (one point per line, in grid
 * index units, scaled by Grid.Stride).  The parser is a self-contained YAML
 * subset reader (block maps and sequences, flow sequences, scalars,
 * comments); yaml-cpp is not needed.
 *
 * Differences from the reference, both deliberate: errors are returned as
 * status codes (the reference throws on unknown enums and ignores unreadable
 * .xyz files), and optional keys extend the schema -- Simulate.Gravity
 * (default 9.80665), Simulate.Transfer (PICFLIP or APIC, default given by
 * the builder call), Grid.Boundary (Reference or Sticky) and
 * Grid.StickyCells.
 */
#ifndef MPM_B200_CONFIG_H_
#define MPM_B200_CONFIG_H_

#include "mpm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mpm_config_group {
    char file[1024];          /* .xyz path as written in the YAML           */
    float mass;               /* per-particle mass                          */
    float velocity[3];
    mpm_material material;
} mpm_config_group;

/* MPM3DConfiguration (include/mpm3d_parser.h:13-33). */
typedef struct mpm_config {
    int32_t ngroups;
    mpm_config_group* groups; /* owned; released by mpm_config_free */
    float origin[3];
    int32_t resolution[3];
    float stride;
    float friction;
    float blend;
    int32_t interpolation;    /* MPM_INTERP_* */
    float dt;
    int32_t offline;          /* Render.Offline (accepted, unused)          */
    char particle_frag_shader[1024];
    /* extensions */
    float gravity;
    int32_t transfer;         /* -1: not given in the file                  */
    int32_t boundary;
    int32_t sticky_cells;
    char base_dir[1024];      /* directory of the YAML file                 */
} mpm_config;

/* parseYAML.  Unknown ConstitutiveModel / Interpolation names return
 * MPM_ERR_PARSE (the reference throws std::runtime_error, mpm3d_parser.cpp:10,17). */
MPM_API mpm_status mpm_config_parse_yaml(const char* path, mpm_config** out);
/* Same, from YAML text in memory (base_dir is used to resolve .xyz paths). */
MPM_API mpm_status mpm_config_parse_yaml_string(const char* text, const char* base_dir, mpm_config** out);
MPM_API mpm_status mpm_config_free(mpm_config* cfg);

/* readXYZFile followed by the builder's scaling by `stride`
 * (src/mpm_solver3d_builder.cu:10-30,44).  *points is 3 * *n floats,
 * released with mpm_free.  A relative path is tried as given, then against
 * base_dir (may be NULL). */
MPM_API mpm_status mpm_read_xyz(const char* path, const char* base_dir, float stride, float** points, size_t* n);
MPM_API void mpm_free(void* p);

/* buildMPMSolver3DFromYAML / buildAPICMPMSolver3DFromYAML: read every
 * group's .xyz, build one material per group, stack the groups in order and
 * create the solver.  transfer = MPM_TRANSFER_PIC_FLIP or MPM_TRANSFER_APIC
 * (a Simulate.Transfer key in the file overrides it when transfer < 0). */
MPM_API mpm_status mpm_solver_create_from_config(const mpm_config* cfg, int32_t transfer, mpm_solver** out,
                                                 int32_t* particles_number);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_CONFIG_H_ */
