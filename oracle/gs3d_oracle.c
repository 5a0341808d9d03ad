/*
 * gs3d_oracle.c -- TEST INFRASTRUCTURE: the CPU oracle for the harmonyos_3dgs
 * 2D render/train path.  Only tests/, the smoke check and bench.py's CPU
 * baseline load this library; the CUDA product path never does.
 *
 * Parity is pinned two ways (see tests/test_oracle_pin.py):
 *   - against the reference's own golden vectors (train/verify_grads_ext/<scene>,
 *     train/verify_forward, tests/test_data/l1_verify), copied as fixtures
 *     under tests/golden/;
 *   - against the reference's CPU stages themselves, compiled from their own
 *     sources into oracle/_ref/ (oracle/Makefile) and run on seeded scenes.
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared (oracle/Makefile).  The
 * float instantiation must not be contracted into FMAs, exactly like the
 * reference build (CMakeLists.txt:19).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gs3d_oracle.h"

#define REAL float
#define SFX(n) n##_f32
#define R_SQRT sqrtf
#define R_EXP expf
#define R_CEIL ceilf
#define R_LOG logf
#define R_POW powf
#include "gs3d_oracle_core.inc"
#undef REAL
#undef SFX
#undef R_SQRT
#undef R_EXP
#undef R_CEIL
#undef R_LOG
#undef R_POW

#define REAL double
#define SFX(n) n##_f64
#define R_SQRT sqrt
#define R_EXP exp
#define R_CEIL ceil
#define R_LOG log
#define R_POW pow
#include "gs3d_oracle_core.inc"
#undef REAL
#undef SFX

/* ---------- 3D evaluation (eval_3D), float only ---------- */
#include "gs3d_oracle_eval3d.inc"

/* ---------- adaptive density control, float only ---------- */
#include "gs3d_oracle_density.inc"

/* ---------- binning: tile_binner_cpu.cpp:33-99 ---------- */

/* Inclusive scan of tiles_touched (:33-42); returns total pairs. */
int64_t orc_scan_tiles(int N, const int* tiles, int64_t* incl) {
    int64_t acc = 0;
    for (int i = 0; i < N; i++) {
        acc += tiles[i];
        if (incl) incl[i] = acc;
    }
    return acc;
}

/* Emits (tile<<32 | depth bits, gaussian index) in Gaussian order, tiles
 * row-major inside each rect (:59-99). keys/vals hold the scan's total. */
void orc_bin(int N, const float* means2D, const float* depths, const int* radii, const int* tiles,
             const gs3d_camera* cam, const gs3d_render_config* cfg, uint64_t* keys, uint32_t* vals) {
    int grid_x = (cam->width + cfg->tile_w - 1) / cfg->tile_w;
    int grid_y = (cam->height + cfg->tile_h - 1) / cfg->tile_h;
    int64_t off = 0;
    for (int i = 0; i < N; i++) {
        int64_t base = off;
        off += tiles[i];
        if (radii[i] <= 0) continue;
        int rmn[2], rmx[2];
        tile_rect_f32(means2D[2 * i], means2D[2 * i + 1], radii[i], grid_x, grid_y, cfg->tile_w,
                      cfg->tile_h, rmn, rmx);
        uint32_t dbits;
        memcpy(&dbits, &depths[i], 4);
        int64_t o = base;
        for (int y = rmn[1]; y < rmx[1]; y++)
            for (int x = rmn[0]; x < rmx[0]; x++) {
                uint32_t tile = (uint32_t)(y * grid_x + x);
                keys[o] = ((uint64_t)tile << 32) | dbits;
                vals[o] = (uint32_t)i;
                o++;
            }
    }
}

/* ---------- sort + ranges: sorter_cpu.cpp:13-43 ---------- */

typedef struct { uint64_t key; uint64_t pos; } orc_kp;

static int orc_kp_cmp(const void* a, const void* b) {
    const orc_kp* x = (const orc_kp*)a;
    const orc_kp* y = (const orc_kp*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos ? 1 : 0);
}

/* Stable sort by key (ties keep input order; the reference's std::sort is
 * unstable, so tests compare values modulo runs of equal keys), then the
 * per-tile [start, end) ranges, zero for empty tiles. */
void orc_sort(int64_t P, const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
              uint32_t* vals_out, int num_tiles, uint32_t* ranges) {
    memset(ranges, 0, (size_t)num_tiles * 2 * sizeof(uint32_t));
    if (P <= 0) return;
    orc_kp* kp = (orc_kp*)malloc((size_t)P * sizeof(orc_kp));
    for (int64_t i = 0; i < P; i++) { kp[i].key = keys_in[i]; kp[i].pos = (uint64_t)i; }
    qsort(kp, (size_t)P, sizeof(orc_kp), orc_kp_cmp);
    for (int64_t i = 0; i < P; i++) {
        keys_out[i] = kp[i].key;
        vals_out[i] = vals_in[kp[i].pos];
    }
    free(kp);
    for (int64_t i = 0; i < P; i++) {
        uint32_t t = (uint32_t)(keys_out[i] >> 32);
        if (i == 0) ranges[2 * t] = 0;
        else {
            uint32_t pt = (uint32_t)(keys_out[i - 1] >> 32);
            if (t != pt) { ranges[2 * pt + 1] = (uint32_t)i; ranges[2 * t] = (uint32_t)i; }
        }
        if (i == P - 1) ranges[2 * t + 1] = (uint32_t)P;
    }
}

/* ---------- composite drivers (trainer.cpp:7-70, renderer.cpp:13-39) ---------- */

/* Forward through rasterisation from an activated model.  Returns 0, or 1
 * when the pair capacity is too small (total_pairs is still set). */
int orc_forward(const gs3d_gaussians* g, const gs3d_camera* cam, const gs3d_render_config* cfg,
                orc_step_io* io) {
    int N = g->count;
    orc_preprocess_f32(N, g->sh_degree, g->max_coeffs, g->positions, g->scales, g->rotations,
                       g->sh_coeffs, g->opacities, cam, cfg, io->means2D, io->depths, io->conics,
                       io->opac2d, io->rgb, io->radii, io->tiles, io->cov3D, io->p_view, io->p_hom_w,
                       io->cov2D, io->det);
    io->total_pairs = orc_scan_tiles(N, io->tiles, NULL);
    if (io->total_pairs > io->pair_capacity) return 1;
    orc_bin(N, io->means2D, io->depths, io->radii, io->tiles, cam, cfg, io->keys_unsorted,
            io->vals_unsorted);
    int grid_x = (cam->width + cfg->tile_w - 1) / cfg->tile_w;
    int grid_y = (cam->height + cfg->tile_h - 1) / cfg->tile_h;
    orc_sort(io->total_pairs, io->keys_unsorted, io->vals_unsorted, io->keys_sorted, io->vals_sorted,
             grid_x * grid_y, io->ranges);
    orc_rasterize_f32(io->means2D, io->conics, io->opac2d, io->rgb, io->vals_sorted, io->ranges, cam,
                      cfg, io->image, io->T_final, io->n_contrib);
    return 0;
}

/* Forward of the 3D-evaluation mode (cfg->eval_3D): the same sequence with
 * the eval_3D preprocess, per-tile depth keys and the buffered blend.
 * g2s[16N], ci[6N], mo[3N] receive the mode's extra per-Gaussian outputs. */
int orc_forward_eval3d(const gs3d_gaussians* g, const gs3d_camera* cam, const gs3d_render_config* cfg,
                       orc_step_io* io, float* g2s, float* ci, float* mo) {
    int N = g->count;
    orc_preprocess_eval3d(g, cam, cfg, io->means2D, io->depths, io->conics, io->opac2d, io->rgb, io->radii,
                          io->tiles, g2s, ci, mo);
    io->total_pairs = orc_scan_tiles(N, io->tiles, NULL);
    if (io->total_pairs > io->pair_capacity) return 1;
    orc_bin_eval3d(N, io->means2D, io->depths, io->radii, io->tiles, ci, mo, cam, cfg, io->keys_unsorted,
                   io->vals_unsorted);
    int grid_x = (cam->width + cfg->tile_w - 1) / cfg->tile_w;
    int grid_y = (cam->height + cfg->tile_h - 1) / cfg->tile_h;
    orc_sort(io->total_pairs, io->keys_unsorted, io->vals_unsorted, io->keys_sorted, io->vals_sorted,
             grid_x * grid_y, io->ranges);
    orc_rasterize_eval3d(g2s, io->opac2d, io->rgb, io->depths, ci, mo, io->vals_sorted, io->ranges, cam, cfg,
                         io->image, io->T_final, io->n_contrib);
    return 0;
}

/* One Trainer::step with use_adam (trainer.cpp:7-70).  raw is updated in
 * place; act_* are scratch for the activated model.  Returns 0, or 1 on a
 * pair-capacity overflow (nothing is updated then). */
int orc_train_step(gs3d_raw_params* raw, const gs3d_camera* cam, const float* gt,
                   const gs3d_render_config* cfg, const gs3d_train_config* tc, int iteration,
                   orc_adam_state* st, float* act_pos, float* act_sc, float* act_rot, float* act_sh,
                   float* act_op, orc_step_io* io) {
    int N = raw->count, mc3 = raw->max_coeffs * 3;
    orc_activate_f32(N, mc3, raw->raw_positions, raw->raw_scales, raw->raw_rotations,
                     raw->raw_sh_coeffs, raw->raw_opacities, act_pos, act_sc, act_rot, act_sh, act_op);
    gs3d_gaussians g = {N, raw->sh_degree, raw->max_coeffs, act_pos, act_sh, act_sc, act_rot, act_op, NULL};
    if (orc_forward(&g, cam, cfg, io)) return 1;
    int H = cam->height, W = cam->width;
    io->loss = orc_l1_loss_f32(io->image, gt, H, W, io->d_image);
    {
        double s = 0;
        int64_t n = (int64_t)H * W * 3;
        for (int64_t i = 0; i < n; i++) s += fabs((double)(io->image[i] - gt[i]));
        io->loss_acc64 = s / (double)n;
    }
    memset(io->d_means2D, 0, sizeof(float) * 2 * N);
    memset(io->d_conics, 0, sizeof(float) * 3 * N);
    memset(io->d_rgb, 0, sizeof(float) * 3 * N);
    memset(io->d_opac, 0, sizeof(float) * N);
    orc_raster_backward_f32(io->means2D, io->conics, io->opac2d, io->rgb, io->vals_sorted, io->ranges,
                            cam, cfg, io->T_final, io->n_contrib, io->d_image, io->d_means2D,
                            io->d_conics, io->d_rgb, io->d_opac);
    memset(io->g_pos, 0, sizeof(float) * 3 * N);
    memset(io->g_sc, 0, sizeof(float) * 3 * N);
    memset(io->g_rot, 0, sizeof(float) * 4 * N);
    memset(io->g_sh, 0, sizeof(float) * (size_t)mc3 * N);
    memset(io->g_op, 0, sizeof(float) * N);
    orc_preprocess_backward_f32(N, raw->sh_degree, raw->max_coeffs, act_pos, act_sc, act_rot, act_sh,
                                act_op, raw->raw_rotations, cam, cfg, io->radii, io->means2D, io->cov3D,
                                io->p_view, io->p_hom_w, io->cov2D, io->det, io->d_means2D,
                                io->d_conics, io->d_rgb, io->d_opac, io->g_pos, io->g_sc, io->g_rot,
                                io->g_sh, io->g_op);
    if (tc->use_adam) {
        st->step_count++;
        float bc1, bc2;
        orc_adam_bias_f32(tc->adam_beta1, tc->adam_beta2, st->step_count, &bc1, &bc2);
        float lr_pos = orc_lr_schedule_f32(tc->lr_position_init, tc->lr_position_final, iteration,
                                           tc->max_steps);
        float b1 = tc->adam_beta1, b2 = tc->adam_beta2, eps = tc->adam_eps;
        orc_adam_update_f32(raw->raw_positions, io->g_pos, st->m_pos, st->v_pos, (int64_t)N * 3, lr_pos,
                            b1, b2, eps, bc1, bc2);
        orc_adam_update_f32(raw->raw_scales, io->g_sc, st->m_sc, st->v_sc, (int64_t)N * 3, tc->lr_scaling,
                            b1, b2, eps, bc1, bc2);
        orc_adam_update_f32(raw->raw_rotations, io->g_rot, st->m_rot, st->v_rot, (int64_t)N * 4,
                            tc->lr_rotation, b1, b2, eps, bc1, bc2);
        orc_adam_update_f32(raw->raw_sh_coeffs, io->g_sh, st->m_sh, st->v_sh, (int64_t)N * mc3,
                            tc->lr_feature, b1, b2, eps, bc1, bc2);
        orc_adam_update_f32(raw->raw_opacities, io->g_op, st->m_op, st->v_op, (int64_t)N, tc->lr_opacity,
                            b1, b2, eps, bc1, bc2);
    } else {
        /* SGD, optimizer.cpp:9-26 */
        float lr_pos = orc_lr_schedule_f32(tc->lr_position_init, tc->lr_position_final, iteration,
                                           tc->max_steps);
        for (int64_t i = 0; i < (int64_t)N * 3; i++) raw->raw_positions[i] -= lr_pos * io->g_pos[i];
        for (int64_t i = 0; i < (int64_t)N * 3; i++) raw->raw_scales[i] -= tc->lr_scaling * io->g_sc[i];
        for (int64_t i = 0; i < (int64_t)N * 4; i++) raw->raw_rotations[i] -= tc->lr_rotation * io->g_rot[i];
        for (int64_t i = 0; i < (int64_t)N * mc3; i++) raw->raw_sh_coeffs[i] -= tc->lr_feature * io->g_sh[i];
        for (int64_t i = 0; i < N; i++) raw->raw_opacities[i] -= tc->lr_opacity * io->g_op[i];
    }
    return 0;
}

/* ---------- FP64 oracle: loss, image and gradients of the same function ---------- */

typedef struct { uint32_t tile; double depth; uint32_t idx; } orc_pair64;

static int orc_pair64_cmp(const void* a, const void* b) {
    const orc_pair64* x = (const orc_pair64*)a;
    const orc_pair64* y = (const orc_pair64*)b;
    if (x->tile != y->tile) return x->tile < y->tile ? -1 : 1;
    if (x->depth != y->depth) return x->depth < y->depth ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx ? 1 : 0);
}

/* FP64 evaluation of the whole step's function from double raw parameters:
 * image, L1 loss (double) and, when grads are non-NULL, the analytic FP64
 * adjoint gradients w.r.t. the raw parameters.  Tiles, culling and the
 * per-tile depth order are decided in FP64 too. */
double orc_step_f64(int N, int sh_degree, int max_coeffs, const double* rpos, const double* rsc,
                    const double* rrot, const double* rsh, const double* rop, const gs3d_camera* cam,
                    const gs3d_render_config* cfg, const float* gt, double* image_out,
                    double* g_pos, double* g_sc, double* g_rot, double* g_sh, double* g_op) {
    int mc3 = max_coeffs * 3;
    int H = cam->height, W = cam->width;
    int64_t npx = (int64_t)H * W;
    double *pos = malloc(sizeof(double) * 3 * N), *sc = malloc(sizeof(double) * 3 * N);
    double *rot = malloc(sizeof(double) * 4 * N), *sh = malloc(sizeof(double) * (size_t)mc3 * N);
    double* op = malloc(sizeof(double) * N);
    orc_activate_f64(N, mc3, rpos, rsc, rrot, rsh, rop, pos, sc, rot, sh, op);
    double *m2 = malloc(sizeof(double) * 2 * N), *dep = malloc(sizeof(double) * N);
    double *con = malloc(sizeof(double) * 3 * N), *o2 = malloc(sizeof(double) * N);
    double* rgb = malloc(sizeof(double) * 3 * N);
    int *rad = malloc(sizeof(int) * N), *tl = malloc(sizeof(int) * N);
    double *c3 = malloc(sizeof(double) * 6 * N), *pv = malloc(sizeof(double) * 3 * N);
    double *pw = malloc(sizeof(double) * N), *c2 = malloc(sizeof(double) * 3 * N);
    double* dt = malloc(sizeof(double) * N);
    orc_preprocess_f64(N, sh_degree, max_coeffs, pos, sc, rot, sh, op, cam, cfg, m2, dep, con, o2, rgb,
                       rad, tl, c3, pv, pw, c2, dt);
    int64_t P = 0;
    for (int i = 0; i < N; i++) P += tl[i];
    int grid_x = (W + cfg->tile_w - 1) / cfg->tile_w, grid_y = (H + cfg->tile_h - 1) / cfg->tile_h;
    int ntiles = grid_x * grid_y;
    orc_pair64* pr = malloc(sizeof(orc_pair64) * (size_t)(P > 0 ? P : 1));
    int64_t o = 0;
    for (int i = 0; i < N; i++) {
        if (rad[i] <= 0) continue;
        int rmn[2], rmx[2];
        tile_rect_f64(m2[2 * i], m2[2 * i + 1], rad[i], grid_x, grid_y, cfg->tile_w, cfg->tile_h, rmn, rmx);
        for (int y = rmn[1]; y < rmx[1]; y++)
            for (int x = rmn[0]; x < rmx[0]; x++) {
                pr[o].tile = (uint32_t)(y * grid_x + x);
                pr[o].depth = dep[i];
                pr[o].idx = (uint32_t)i;
                o++;
            }
    }
    qsort(pr, (size_t)P, sizeof(orc_pair64), orc_pair64_cmp);
    uint32_t* vs = malloc(sizeof(uint32_t) * (size_t)(P > 0 ? P : 1));
    uint32_t* rg = calloc((size_t)ntiles * 2, sizeof(uint32_t));
    for (int64_t i = 0; i < P; i++) {
        vs[i] = pr[i].idx;
        uint32_t t = pr[i].tile;
        if (i == 0 || pr[i - 1].tile != t) rg[2 * t] = (uint32_t)i;
        rg[2 * t + 1] = (uint32_t)(i + 1);
    }
    double* img = image_out ? image_out : malloc(sizeof(double) * 3 * npx);
    double* Tf = malloc(sizeof(double) * npx);
    int* nc = malloc(sizeof(int) * npx);
    orc_rasterize_f64(m2, con, o2, rgb, vs, rg, cam, cfg, img, Tf, nc);
    double* gtd = malloc(sizeof(double) * 3 * npx);
    for (int64_t i = 0; i < 3 * npx; i++) gtd[i] = gt ? (double)gt[i] : 0.0;
    double* dimg = g_pos ? malloc(sizeof(double) * 3 * npx) : NULL;
    double loss = orc_l1_loss_f64(img, gtd, H, W, dimg);
    if (g_pos) {
        /* d_image = sign(diff)/n evaluated in FP64 (the float form uses 1.0f/n) */
        double inv_n = 1.0 / (double)(3 * npx);
        for (int64_t i = 0; i < 3 * npx; i++) {
            double d = img[i] - gtd[i];
            dimg[i] = d > 0 ? inv_n : (d < 0 ? -inv_n : 0.0);
        }
        double *dm = calloc((size_t)2 * N, sizeof(double)), *dc = calloc((size_t)3 * N, sizeof(double));
        double *dr = calloc((size_t)3 * N, sizeof(double)), *dop = calloc((size_t)N, sizeof(double));
        orc_raster_backward_f64(m2, con, o2, rgb, vs, rg, cam, cfg, Tf, nc, dimg, dm, dc, dr, dop);
        memset(g_pos, 0, sizeof(double) * 3 * N);
        memset(g_sc, 0, sizeof(double) * 3 * N);
        memset(g_rot, 0, sizeof(double) * 4 * N);
        memset(g_sh, 0, sizeof(double) * (size_t)mc3 * N);
        memset(g_op, 0, sizeof(double) * N);
        orc_preprocess_backward_f64(N, sh_degree, max_coeffs, pos, sc, rot, sh, op, rrot, cam, cfg, rad,
                                    m2, c3, pv, pw, c2, dt, dm, dc, dr, dop, g_pos, g_sc, g_rot, g_sh,
                                    g_op);
        free(dm); free(dc); free(dr); free(dop);
        free(dimg);
    }
    free(pos); free(sc); free(rot); free(sh); free(op);
    free(m2); free(dep); free(con); free(o2); free(rgb); free(rad); free(tl);
    free(c3); free(pv); free(pw); free(c2); free(dt);
    free(pr); free(vs); free(rg);
    if (!image_out) free(img);
    free(Tf); free(nc); free(gtd);
    return loss;
}
