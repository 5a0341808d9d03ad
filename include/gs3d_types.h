/*
 * gs3d_types.h -- plain-C restatement of the buffer layouts that the
 * harmonyos_3dgs render/train path passes between its stages.
 *
 * Every struct here is byte-for-byte layout-identical to the reference's C++
 * struct of the same role, so a caller holding the reference type passes it
 * across the C ABI with a reinterpret_cast and no copy.  The C++ adapter
 * (aaags_claude_b200/host/gs3d_stages_cuda.cpp) static_asserts sizeof and
 * every offsetof against the reference headers when it is compiled with them.
 *
 *   gs3d_gaussians      <-> GaussianData       include/types.h:34-45
 *   gs3d_camera         <-> Camera             include/types.h:48-54
 *   gs3d_render_config  <-> RenderConfig       include/types.h:57-66
 *   gs3d_raw_params     <-> RawGaussianParams  include/train_types.h:9-22
 *   gs3d_train_config   <-> TrainConfig        include/train_types.h:46-60
 *   gs3d_densify_config <-> DensifyConfig      include/train_types.h:70-81
 *
 * Conventions kept from the reference:
 *   - all matrices are 4x4 column-major (GLM order);
 *   - SH coefficients are [N][max_coeffs][3], RGB interleaved per basis;
 *   - quaternions are (r, x, y, z);
 *   - images are H x W x 3 (HWC) float;
 *   - tile binning keys are (uint64_t)tile_id << 32 | float_bits(view depth).
 */
#ifndef GS3D_TYPES_H
#define GS3D_TYPES_H

#include <stdint.h>
#include <stddef.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Activated (post exp/normalize/sigmoid) model, structure of arrays. */
typedef struct gs3d_gaussians {
    int count;            /* N */
    int sh_degree;        /* 0..3 */
    int max_coeffs;       /* (sh_degree+1)^2 */
    float* positions;     /* [N*3] world xyz */
    float* sh_coeffs;     /* [N*max_coeffs*3] */
    float* scales;        /* [N*3] exp()-activated */
    float* rotations;     /* [N*4] unit quaternion (r,x,y,z) */
    float* opacities;     /* [N] sigmoid()-activated */
    float* filter_3D;     /* [N] or NULL: 3D mip filter of the eval_3D mode */
} gs3d_gaussians;

/* Pinhole camera: world->view and world->clip, both column-major. */
typedef struct gs3d_camera {
    float view_matrix[16];
    float viewproj_matrix[16];
    float cam_pos[3];
    float tan_fovx, tan_fovy;
    int width, height;
} gs3d_camera;

/* Render options; the reference's C++ defaults are bg 0, scale 1, sh 3, 16x16 tiles. */
typedef struct gs3d_render_config {
    float bg_color[3];
    float scale_modifier;
    bool antialiasing;
    bool eval_3D;         /* AAA-Gaussians 3D evaluation: render calls only (no backward) */
    bool training;        /* true: no upper clamp on SH colour */
    int sh_degree;
    int tile_w;
    int tile_h;
} gs3d_render_config;

/* Raw (pre-activation) trainable parameters. */
typedef struct gs3d_raw_params {
    int count;
    int sh_degree;
    int max_coeffs;
    float* raw_positions;  /* [N*3] identity */
    float* raw_scales;     /* [N*3] log scale */
    float* raw_rotations;  /* [N*4] unnormalised quaternion */
    float* raw_sh_coeffs;  /* [N*max_coeffs*3] identity */
    float* raw_opacities;  /* [N] logit */
} gs3d_raw_params;

/* Optimiser hyper-parameters (Adam when use_adam, else SGD). */
typedef struct gs3d_train_config {
    float lr_position_init;
    float lr_position_final;
    float lr_feature;
    float lr_opacity;
    float lr_scaling;
    float lr_rotation;
    int max_steps;
    bool use_adam;
    float adam_beta1;
    float adam_beta2;
    float adam_eps;
} gs3d_train_config;

/* Adaptive density control (clone / split / prune, opacity reset). */
typedef struct gs3d_densify_config {
    int densify_from_iter;      /* 500 */
    int densify_until_iter;     /* 15000 */
    int densify_interval;       /* 100 */
    float grad_threshold;       /* 0.0002 */
    float min_opacity;          /* 0.005 */
    float percent_dense;        /* 0.01 (the reference's controller uses 0.01 whatever this holds) */
    int opacity_reset_interval; /* 3000 */
    int max_screen_size;        /* 20 */
    bool enabled;               /* false: opt-in */
} gs3d_densify_config;

#ifdef __cplusplus
}
#endif

#endif /* GS3D_TYPES_H */
