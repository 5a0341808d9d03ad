/*
 * gs3d_oracle.h -- TEST INFRASTRUCTURE.  Declarations shared by the C oracle
 * (gs3d_oracle.c) and the shim over the reference's own CPU stages
 * (ref_shim.cpp, built into oracle/_ref/).  Both fill the same I/O struct so
 * tests compare them field by field.
 */
#ifndef GS3D_ORACLE_H
#define GS3D_ORACLE_H

#include <stdint.h>
#include "../include/gs3d_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_step_io {
    float *means2D, *depths, *conics, *opac2d, *rgb;
    int *radii, *tiles;
    float *cov3D, *p_view, *p_hom_w, *cov2D, *det;
    int64_t pair_capacity, total_pairs;
    uint64_t *keys_unsorted, *keys_sorted;
    uint32_t *vals_unsorted, *vals_sorted, *ranges;
    float *image, *T_final;
    int* n_contrib;
    float* d_image;
    float *d_means2D, *d_conics, *d_rgb, *d_opac;
    float *g_pos, *g_sc, *g_rot, *g_sh, *g_op;
    float loss;
    double loss_acc64;
} orc_step_io;

typedef struct orc_adam_state {
    float *m_pos, *v_pos, *m_sc, *v_sc, *m_rot, *v_rot, *m_sh, *v_sh, *m_op, *v_op;
    int step_count;
} orc_adam_state;

#ifdef __cplusplus
}
#endif

#endif
