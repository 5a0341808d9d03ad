// capi.cu -- the gs3dc_* C ABI (include/gs3d_cuda.h): context, device buffers,
// stage entry points and the graph-replayed train step.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gs3d_cuda.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace gs3d;

namespace {

// Bumped by every device (re)allocation of a context buffer that captured
// launches address: a captured graph holds buffer addresses, so the graph
// cache keys include this epoch and a graph captured before any reallocation
// is never replayed after it.
std::atomic<unsigned long long> g_alloc_epoch{1};

// A device buffer that only grows.  kGraphAddressed = false: no captured launch
// holds its address (buffers reached through the per-step parameter block,
// such as the host targets' device copies), so reallocating it keeps graphs.
template <class T, bool kGraphAddressed = true>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t need) {
        if (need <= n && p) return cudaSuccess;
        if (kGraphAddressed) g_alloc_epoch.fetch_add(1, std::memory_order_relaxed);
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (need == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, need * sizeof(T));
        if (e == cudaSuccess) n = need;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p && kGraphAddressed) g_alloc_epoch.fetch_add(1, std::memory_order_relaxed);
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

constexpr int kParamSlots = 4;  // pinned ring of per-step parameter blocks
constexpr int kMaxBatchViews = 255;   // views per multi-view step (one 8-bit radix digit)
constexpr int kTunePpt[3] = {1, 2, 4};   // autotuner candidates: pixels per thread of the rasterisers
constexpr int kTuneBatch[2] = {64, 256}; // then: records staged per round (against the default 128)
constexpr int kTuneReps = 2;             // timed steps per candidate
constexpr int kTunePptSteps = 3 * kTuneReps;
constexpr int kTuneSteps = kTunePptSteps + 2 * kTuneReps;
constexpr int kShapeSlots = 8;           // single-view train step: workload shapes with a cached graph / tuning
constexpr int kGraphKey = 9;             // words of a graph key

}  // namespace

struct gs3dc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;

    // model (raw when model_raw, else activated)
    int N = 0, sh_degree = 0, max_coeffs = 1;
    bool have_model = false, model_raw = false;
    DevBuf<float> pos, sc, rot, sh, op;
    // Adam moments + stand-alone gradients
    DevBuf<float> m_pos, v_pos, m_sc, v_sc, m_rot, v_rot, m_sh, v_sh, m_op, v_op;
    DevBuf<float> g_pos, g_sc, g_rot, g_sh, g_op;
    int adam_step = 0;
    // screen-space records + optional cache
    DevBuf<float4> rec0, rec1;
    DevBuf<float2> cbt;
    DevBuf<float> depth;
    DevBuf<int> radius, tiles;
    DevBuf<float> c_cov3D, c_pview, c_phw, c_cov2D, c_det;
    // screen arrays in the reference layout (stage import / export)
    DevBuf<float> x_means2D, x_depths, x_conics, x_opac, x_rgb;
    DevBuf<int> x_radii, x_tiles;
    // raster gradients
    DevBuf<float> dm2, dcon, drgb, dop;
    // pairs
    DevBuf<unsigned long long> keys[2];
    DevBuf<unsigned> vals[2];
    unsigned long long cap = 0, min_cap = 0;
    int sorted_which = 0;
    DevBuf<unsigned long long> sort_desc;
    unsigned long long sort_desc_stride = 0;
    int sort_passes = 0, sort_num_tiles = 0;
    // depth-first ordering of the train step: Gaussian depth sort buffers
    int sort_mode = GS3DC_SORT_DEPTH_FIRST;
    DevBuf<unsigned> dkeys[2];
    DevBuf<unsigned> dvals[2];
    DevBuf<unsigned long long> ddesc;
    unsigned long long ddesc_stride = 0;
    // reduced-storage form (GS3DC_FORM_BF16 / _FP16); the FP32 model arrays above stage uploads
    int form = GS3DC_FORM_PLAIN_FP32;
    bool chosen_ready = false;   // the chosen buffers hold the current model
    DevBuf<float> c_pos, cm_pos, cv_pos;
    DevBuf<unsigned short> c_attr, c_sh, cm_attr, cv_attr, cm_sh, cv_sh;
    DevBuf<uint2> c_rects;   // per-Gaussian tile rectangles read by the depth-first pair emission (both forms)
    // 3D-evaluation mode (RenderConfig::eval_3D): per-Gaussian records, tile rays, view
    DevBuf<float4> e3_rec, e3_tdir;
    DevBuf<float> e3_g2s, e3_ci, e3_mo, e3_view, filt3d;
    bool have_filt3d = false;   // the activated model came with GaussianData::filter_3D
    bool mode_e3 = false;       // the current screen records and pairs are of the 3D mode
    int screen_n = 0;             // Gaussians of the current screen records
    bool screen_imported = false; // the screen records came from a caller (gs3dc_rasterize_arrays)
    // adaptive density control (the trainer's DensityController): statistics + scratch
    DevBuf<float> dc_accum, dc_denom;
    DevBuf<int> dc_maxr, dc_clone, dc_split, dc_crank, dc_srank, dc_src, dc_keep, dc_out, dc_sums, dc_radii_in;
    DevBuf<float> dc_dm_in;              // host d_means2D uploaded by gs3dc_density_accumulate
    DevBuf<float> dc_t[5], dc_new[5];   // post-split and final parameter arrays (pos, sc, rot, sh, op)
    int dc_n = 0;                        // Gaussians the statistics describe
    unsigned long long dc_rng = 12345ull;   // the split sampler's LCG state (density_controller.h)
    // control block + preprocess scan descriptors (one memset)
    DevBuf<unsigned char> ctrl_region;
    Control* ctrl = nullptr;
    unsigned long long* scan_desc = nullptr;
    Control* ctrl_host = nullptr;  // pinned readback
    // tiles / pixels
    int W = 0, H = 0, num_tiles = 0;
    DevBuf<unsigned> ranges;
    DevBuf<unsigned> tile_order;   // heavy-first permutation of the tiles
    DevBuf<float> image, T_final, d_image, gt;
    DevBuf<float> raw_rot_tmp;   // raw quaternions for the backward of an activated model
    DevBuf<int> n_contrib;
    DevBuf<unsigned> last_j;
    DevBuf<unsigned char> dsign;
    // stored-list raster backward (gs3dc_raster_backward_lists): per-pixel entry offsets and the lists
    DevBuf<int> list_off;
    DevBuf<uint2> lists;
    // per-step parameters: device copy + pinned ring
    StepParams* sp_dev = nullptr;
    Persist* persist = nullptr;       // device
    Persist* persist_host = nullptr;  // pinned readback
    StepParams* sp_ring = nullptr;
    cudaEvent_t sp_event[kParamSlots] = {};
    int sp_slot = 0;
    // stage state
    bool have_screen = false, have_pairs = false, have_sorted = false, have_raster = false,
         have_rgrad = false, have_grads = false;
    // graph of the train step
    bool use_graph = true;
    bool fused_adam = false;   // split backward + optimiser by default (faster at this occupancy)
    bool keep_grads = false;   // GS3DC_OPT_KEEP_GRADIENTS
    bool have_step_grads = false;
    // captured single-view steps, one slot per workload shape (least recently used replaced): a
    // caller alternating between camera sizes replays each size's graphs instead of re-capturing
    struct GraphSlot {
        long long key[kGraphKey] = {};
        cudaGraphExec_t front = nullptr;   // preprocess .. tile ranges
        cudaGraphExec_t back = nullptr;    // rasterisers, backward, optimiser
        long long kernels = 0;
        unsigned long long used = 0;       // LRU clock of the last replay
    };
    GraphSlot gslots[kShapeSlots];
    unsigned long long gclock = 0;
    long long graph_captures = 0;
    // shapes whose pair capacity a synchronous step has validated (N, SH width, W, H, form, order)
    long long seen_shape[kShapeSlots][6] = {};
    int seen_next = 0;
    // host targets: copied on their own stream into alternating buffers while the front half runs
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_gt_ready = nullptr;
    cudaEvent_t ev_gt_free[2] = {};
    bool gt_free_recorded[2] = {false, false};
    int gt_slot = 0;
    DevBuf<float, false> gtb[2];   // read through StepParams::gt
    long long graph_replays = 0;
    bool pending_check = false;
    // stage timing
    bool stage_timing = false;
    cudaEvent_t stage_ev[GS3DC_NUM_STAGES + 1] = {};
    float stage_ms[GS3DC_NUM_STAGES] = {};
    // multi-view train step (gs3dc_train_step_batch): (view, Gaussian) entries view * N + i
    struct Batch {
        DevBuf<StepParams> views;                  // per-view parameters (device)
        StepParams* views_host = nullptr;          // pinned staging, kMaxBatchViews entries
        cudaEvent_t views_event = nullptr;         // the staging's last copy has been consumed
        DevBuf<float4> rec0, rec1;
        DevBuf<float2> cbt;
        DevBuf<float> dm2, dcon, drgb, dop;
        DevBuf<uint2> rects;
        DevBuf<unsigned> dkeys[2];                 // (view << 24 | depth's upper 24 bits) of each entry
        DevBuf<unsigned> dvals[2];
        DevBuf<unsigned long long> ddesc, sort_desc;
        DevBuf<unsigned> keys[2], vals[2];
        unsigned long long cap = 0;
        DevBuf<float> image, T;
        DevBuf<float, false> gt;                   // read through the views' StepParams::gt
        DevBuf<unsigned> last;
        DevBuf<unsigned char> dsign;
        DevBuf<unsigned> ranges, order;
        DevBuf<unsigned> hist_parts;               // launch_emit_ranked's spread tile-digit counts
        DevBuf<unsigned> seg_hist;                 // per-view digit counts of the depth sort
        size_t grads_zeroed = 0;                   // entries of the screen-gradient accumulators known zero
        std::vector<unsigned long long> view_pix;  // first pixel of each view of the last step (+ the total)
        cudaGraphExec_t graph = nullptr;
        long long key[kGraphKey] = {};
    } batch;
    // rasteriser pixels per thread and staging batch in use (set per step; 2 and 128 unless the
    // autotuner chose otherwise)
    int fwd_ppt = 2, bwd_ppt = 2, fwd_batch = 128, bwd_batch = 128;
    // online autotuner (GS3DC_OPT_AUTOTUNE): per workload shape, the first kTuneSteps train steps
    // time both rasterisers, first at each candidate pixels-per-thread (batch 128), then at the
    // fastest ones with each other staging batch; the fastest settings stay
    struct Tune {
        long long key[6] = {};
        int trial = 0;
        float fwd_ms[3] = {}, bwd_ms[3] = {};     // per pixels-per-thread candidate, batch 128
        float fwd_bms[2] = {}, bwd_bms[2] = {};   // per other batch, at the picked pixels per thread
        int fwd_ppt = 2, bwd_ppt = 2, fwd_batch = 128, bwd_batch = 128;
        bool done = false;
        unsigned long long used = 0;   // LRU clock (single-view shapes)
    };
    bool autotune = false;
    int forced_ppt = 0;     // GS3DC_OPT_RASTER_PPT
    int forced_batch = 0;   // GS3DC_OPT_RASTER_BATCH
    Tune tune_single[kShapeSlots], tune_batch;
    unsigned long long tclock = 0;
    cudaEvent_t tune_ev[3] = {};
    // options / stats
    unsigned spin_limit = 1u << 22;
    long long kernels_last = 0;
    unsigned long long last_pairs = 0;
};

namespace {

int fail(gs3dc_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

void drop_slot(gs3dc_ctx::GraphSlot& s) {
    if (s.front) cudaGraphExecDestroy(s.front);
    if (s.back) cudaGraphExecDestroy(s.back);
    s = gs3dc_ctx::GraphSlot();
}

void drop_graphs(gs3dc_ctx* c) {
    for (auto& s : c->gslots) drop_slot(s);
    if (c->batch.graph) cudaGraphExecDestroy(c->batch.graph);
    c->batch.graph = nullptr;
}

// The slot holding graphs captured under `key`, or nullptr.
gs3dc_ctx::GraphSlot* find_slot(gs3dc_ctx* c, const long long key[kGraphKey]) {
    for (auto& s : c->gslots)
        if (s.front && std::memcmp(s.key, key, sizeof(s.key)) == 0) return &s;
    return nullptr;
}

// An empty slot, else the least recently replayed one (its graphs destroyed).
gs3dc_ctx::GraphSlot* victim_slot(gs3dc_ctx* c) {
    gs3dc_ctx::GraphSlot* v = &c->gslots[0];
    for (auto& s : c->gslots) {
        if (!s.front) return &s;
        if (s.used < v->used) v = &s;
    }
    drop_slot(*v);
    return v;
}

bool shape_seen(const gs3dc_ctx* c, const long long shape[6]) {
    for (const auto& s : c->seen_shape)
        if (std::memcmp(s, shape, sizeof(s)) == 0) return true;
    return false;
}

void mark_shape_seen(gs3dc_ctx* c, const long long shape[6]) {
    if (shape_seen(c, shape)) return;
    std::memcpy(c->seen_shape[c->seen_next], shape, sizeof(c->seen_shape[0]));
    c->seen_next = (c->seen_next + 1) % kShapeSlots;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            if (e_ == cudaErrorMemoryAllocation)                                                  \
                return fail(c, GS3DC_ERR_OUT_OF_MEMORY, "%s: %s", #call, cudaGetErrorString(e_)); \
            return fail(c, GS3DC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));              \
        }                                                                                         \
    } while (0)

int bit_length(unsigned v) {
    int b = 0;
    while (v) {
        b++;
        v >>= 1;
    }
    return b;
}

// Key bits to sort: 32 depth bits + enough bits for tile ids < num_tiles.
int sort_passes_for(int num_tiles) {
    const int bits = 32 + bit_length(num_tiles > 1 ? (unsigned)(num_tiles - 1) : 0u);
    return (bits + 7) / 8;
}

ModelPtrs model_ptrs(gs3dc_ctx* c) { return {c->pos.p, c->sc.p, c->rot.p, c->sh.p, c->op.p}; }
AdamPtrs adam_ptrs(gs3dc_ctx* c) {
    return {c->m_pos.p, c->v_pos.p, c->m_sc.p, c->v_sc.p, c->m_rot.p,
            c->v_rot.p, c->m_sh.p,  c->v_sh.p,  c->m_op.p, c->v_op.p};
}
GradPtrs grad_ptrs(gs3dc_ctx* c) { return {c->g_pos.p, c->g_sc.p, c->g_rot.p, c->g_sh.p, c->g_op.p}; }
RGradPtrs rgrad_ptrs(gs3dc_ctx* c) { return {c->dm2.p, c->dcon.p, c->drgb.p, c->dop.p}; }
ScreenPtrs screen_ptrs(gs3dc_ctx* c, bool cache) {
    ScreenPtrs s{c->rec0.p, c->rec1.p, c->cbt.p, c->depth.p, c->radius.p, c->tiles.p,
                 nullptr, nullptr, nullptr, nullptr, nullptr};
    if (cache) {
        s.cov3D = c->c_cov3D.p;
        s.p_view = c->c_pview.p;
        s.p_hom_w = c->c_phw.p;
        s.cov2D = c->c_cov2D.p;
        s.det = c->c_det.p;
    }
    return s;
}
PixelPtrs pixel_ptrs(gs3dc_ctx* c) {
    return {c->image.p, c->T_final.p, c->n_contrib.p, c->last_j.p, c->dsign.p, c->d_image.p};
}

// eval_3D (the reference's AAA-Gaussians mode) renders only: the reference has
// no backward for it and its train drivers set it false (train_main.cpp:495).
int check_config(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg, bool render_only = false) {
    if (!cam || !cfg) return fail(c, GS3DC_ERR_INVALID_ARG, "camera and render config are required");
    if (cam->width <= 0 || cam->height <= 0)
        return fail(c, GS3DC_ERR_INVALID_ARG, "bad image size %dx%d", cam->width, cam->height);
    if (cfg->tile_w != kTile || cfg->tile_h != kTile)
        return fail(c, GS3DC_ERR_INVALID_ARG, "tile size %dx%d: this path is built for 16x16 tiles",
                    cfg->tile_w, cfg->tile_h);
    if (cfg->eval_3D && !render_only)
        return fail(c, GS3DC_ERR_INVALID_ARG, "eval_3D renders only: the 3D-evaluation mode has no backward");
    return GS3DC_OK;
}

// Control block + one look-back descriptor per 256-Gaussian CTA.
int ensure_ctrl(gs3dc_ctx* c, int N) {
    const size_t blocks = std::max<size_t>(2, ((size_t)N + kBlock - 1) / kBlock);
    const size_t head = ((sizeof(Control) + 255) / 256) * 256;
    const size_t bytes = head + (blocks + 1) * sizeof(unsigned long long);
    if (bytes > c->ctrl_region.n) {
        CK(c->ctrl_region.ensure(bytes));
        CK(cudaMemset(c->ctrl_region.p, 0, bytes));
    }
    c->ctrl = reinterpret_cast<Control*>(c->ctrl_region.p);
    c->scan_desc = reinterpret_cast<unsigned long long*>(c->ctrl_region.p + head);
    return GS3DC_OK;
}

// Per-Gaussian buffers for N Gaussians with mc SH bases.
int ensure_model(gs3dc_ctx* c, int N, int mc) {
    const size_t n = (size_t)N;
    CK(c->pos.ensure(3 * n));
    CK(c->sc.ensure(3 * n));
    CK(c->rot.ensure(4 * n));
    CK(c->sh.ensure(3 * n * mc));
    CK(c->op.ensure(n));
    CK(c->rec0.ensure(n));
    CK(c->rec1.ensure(n));
    CK(c->cbt.ensure(n));
    CK(c->depth.ensure(n));
    CK(c->radius.ensure(n));
    CK(c->tiles.ensure(n));
    CK(c->dm2.ensure(2 * n));
    CK(c->dcon.ensure(3 * n));
    CK(c->drgb.ensure(3 * n));
    CK(c->dop.ensure(n));
    return ensure_ctrl(c, N);
}

int ensure_adam(gs3dc_ctx* c) {
    const size_t n = (size_t)c->N, mc3 = (size_t)c->max_coeffs * 3;
    DevBuf<float>* bufs[10] = {&c->m_pos, &c->v_pos, &c->m_sc, &c->v_sc, &c->m_rot,
                               &c->v_rot, &c->m_sh,  &c->v_sh,  &c->m_op, &c->v_op};
    const size_t sizes[10] = {3 * n, 3 * n, 3 * n, 3 * n, 4 * n, 4 * n, mc3 * n, mc3 * n, n, n};
    for (int k = 0; k < 10; k++) CK(bufs[k]->ensure(sizes[k]));
    return GS3DC_OK;
}

int zero_adam(gs3dc_ctx* c) {
    DevBuf<float>* bufs[10] = {&c->m_pos, &c->v_pos, &c->m_sc, &c->v_sc, &c->m_rot,
                               &c->v_rot, &c->m_sh,  &c->v_sh,  &c->m_op, &c->v_op};
    for (int k = 0; k < 10; k++)
        if (bufs[k]->n) CK(cudaMemsetAsync(bufs[k]->p, 0, bufs[k]->n * sizeof(float), c->stream));
    CK(cudaMemsetAsync(c->persist, 0, sizeof(Persist), c->stream));
    c->adam_step = 0;
    return GS3DC_OK;
}

bool chosen_form(const gs3dc_ctx* c) { return c->form != GS3DC_FORM_PLAIN_FP32; }

ChosenPtrs chosen_ptrs(gs3dc_ctx* c) {
    return {c->c_pos.p, c->c_attr.p, c->c_sh.p, c->cm_pos.p, c->cv_pos.p,
            c->cm_attr.p, c->cv_attr.p, c->cm_sh.p, c->cv_sh.p};
}

// Reduced-storage buffers for the current N and SH width, filled from the FP32
// model arrays (round to nearest), optimiser state zeroed.
int load_chosen(gs3dc_ctx* c) {
    const size_t n = (size_t)c->N, mc3 = (size_t)c->max_coeffs * 3;
    CK(c->c_pos.ensure(3 * n));
    CK(c->cm_pos.ensure(3 * n));
    CK(c->cv_pos.ensure(3 * n));
    CK(c->c_attr.ensure(8 * n));
    CK(c->cm_attr.ensure(8 * n));
    CK(c->cv_attr.ensure(8 * n));
    CK(c->c_sh.ensure(mc3 * n));
    CK(c->cm_sh.ensure(mc3 * n));
    CK(c->cv_sh.ensure(mc3 * n));
    CK(c->c_rects.ensure(n ? n : 1));
    if (n) {
        CK(launch_chosen_from_raw(c->stream, c->N, (int)mc3, c->form == GS3DC_FORM_FP16,
                                  ModelPtrs{c->pos.p, c->sc.p, c->rot.p, c->sh.p, c->op.p}, chosen_ptrs(c)));
        CK(cudaMemsetAsync(c->cm_pos.p, 0, 3 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->cv_pos.p, 0, 3 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->cm_attr.p, 0, 8 * n * 2, c->stream));
        CK(cudaMemsetAsync(c->cv_attr.p, 0, 8 * n * 2, c->stream));
        CK(cudaMemsetAsync(c->cm_sh.p, 0, mc3 * n * 2, c->stream));
        CK(cudaMemsetAsync(c->cv_sh.p, 0, mc3 * n * 2, c->stream));
    }
    c->chosen_ready = true;
    return GS3DC_OK;
}

// The reduced-storage model back into the FP32 model arrays.
int unload_chosen(gs3dc_ctx* c) {
    if (!c->chosen_ready || c->N <= 0) return GS3DC_OK;
    CK(launch_chosen_to_raw(c->stream, c->N, c->max_coeffs * 3, c->form == GS3DC_FORM_FP16, chosen_ptrs(c),
                            ModelPtrs{c->pos.p, c->sc.p, c->rot.p, c->sh.p, c->op.p}));
    return GS3DC_OK;
}

int require_plain(gs3dc_ctx* c, const char* what) {
    if (chosen_form(c)) return fail(c, GS3DC_ERR_STATE, "%s needs GS3DC_FORM_PLAIN_FP32", what);
    return GS3DC_OK;
}

int ensure_grads(gs3dc_ctx* c) {
    const size_t n = (size_t)c->N, mc3 = (size_t)c->max_coeffs * 3;
    CK(c->g_pos.ensure(3 * n));
    CK(c->g_sc.ensure(3 * n));
    CK(c->g_rot.ensure(4 * n));
    CK(c->g_sh.ensure(mc3 * n));
    CK(c->g_op.ensure(n));
    return GS3DC_OK;
}

int ensure_cache(gs3dc_ctx* c) {
    const size_t n = (size_t)c->N;
    CK(c->c_cov3D.ensure(6 * n));
    CK(c->c_pview.ensure(3 * n));
    CK(c->c_phw.ensure(n));
    CK(c->c_cov2D.ensure(3 * n));
    CK(c->c_det.ensure(n));
    return GS3DC_OK;
}

int ensure_pixels(gs3dc_ctx* c, int W, int H) {
    const size_t np = (size_t)W * H;
    const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
    CK(c->ranges.ensure(2 * (size_t)gx * gy));
    CK(c->tile_order.ensure((size_t)gx * gy));
    CK(c->image.ensure(3 * np));
    CK(c->T_final.ensure(np));
    CK(c->n_contrib.ensure(np));
    CK(c->last_j.ensure(np));
    CK(c->dsign.ensure(np));
    c->W = W;
    c->H = H;
    c->num_tiles = gx * gy;
    return GS3DC_OK;
}

E3Ptrs e3_ptrs(gs3dc_ctx* c) { return {c->e3_rec.p, c->e3_g2s.p, c->e3_ci.p, c->e3_mo.p, c->e3_tdir.p, c->e3_view.p}; }

// Buffers of the 3D-evaluation mode for N Gaussians and the current tiles.
int ensure_e3(gs3dc_ctx* c, int N) {
    const size_t n = N > 0 ? (size_t)N : 1;
    CK(c->e3_rec.ensure((size_t)kE3Rec * n));
    CK(c->e3_g2s.ensure(16 * n));
    CK(c->e3_ci.ensure(6 * n));
    CK(c->e3_mo.ensure(3 * n));
    CK(c->e3_tdir.ensure(c->num_tiles > 0 ? (size_t)c->num_tiles : 1));
    CK(c->e3_view.ensure(32));
    return GS3DC_OK;
}

// Pair buffers and sort descriptors for `cap` pairs and `num_tiles` tiles.
int ensure_pairs(gs3dc_ctx* c, unsigned long long cap, int num_tiles) {
    if (cap < 4096) cap = 4096;
    if (cap > 0xFFFFFFFFull)
        return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "%llu tile pairs exceed the 32-bit tile-range format", cap);
    if (cap > c->cap) {
        for (int b = 0; b < 2; b++) {
            CK(c->keys[b].ensure(cap));
            CK(c->vals[b].ensure(cap));
        }
        c->cap = cap;
    }
    const int passes = sort_passes_for(num_tiles);
    const unsigned long long stride = ((c->cap + kSortTile - 1) / kSortTile) * 256ull;
    CK(c->sort_desc.ensure((size_t)(passes > 2 ? passes : 2) * stride));
    c->sort_desc_stride = stride;
    c->sort_passes = passes;
    c->sort_num_tiles = num_tiles;
    return GS3DC_OK;
}

// The per-step parameters of one camera.
void fill_params(gs3dc_ctx* c, StepParams& p, const gs3d_camera* cam, const gs3d_render_config* cfg,
                 const gs3d_train_config* tc, int iteration, const float* gt_dev, const float* raw_rot_dev) {
    std::memset(&p, 0, sizeof(p));
    p.cam = *cam;
    p.cfg = *cfg;
    // preprocessor_cpu.cpp:50-53
    p.focal_x = (float)cam->width / (2.0f * cam->tan_fovx);
    p.focal_y = (float)cam->height / (2.0f * cam->tan_fovy);
    p.grid_x = (cam->width + cfg->tile_w - 1) / cfg->tile_w;
    p.grid_y = (cam->height + cfg->tile_h - 1) / cfg->tile_h;
    p.num_tiles = p.grid_x * p.grid_y;
    p.sh_deg_model = c->sh_degree;
    p.sh_deg_fwd = cfg->sh_degree < c->sh_degree ? cfg->sh_degree : c->sh_degree;
    p.max_coeffs = c->max_coeffs;
    p.num_gaussians = c->N;
    p.num_pixels = cam->width * cam->height;
    p.inv_n = 1.0f / (float)(cam->width * cam->height * 3);  // loss.cpp:6
    p.spin_limit = c->spin_limit;
    p.sort_passes = sort_passes_for(p.num_tiles);
    p.sort_bits = 32 + bit_length(p.num_tiles > 1 ? (unsigned)(p.num_tiles - 1) : 0u);
    p.gt = gt_dev;
    p.persist = c->persist;
    p.raw_rot = raw_rot_dev;
    p.seed = (unsigned)iteration * 2654435761u + (unsigned)c->adam_step * 40503u + 1u;
    if (tc) {
        p.use_adam = tc->use_adam ? 1 : 0;
        // lr_schedule, train_types.cpp:64-68
        float t = (float)iteration / (float)tc->max_steps;
        t = std::max(0.0f, std::min(1.0f, t));
        p.lr_pos = std::exp(std::log(tc->lr_position_init) * (1.0f - t) + std::log(tc->lr_position_final) * t);
        p.lr_scale = tc->lr_scaling;
        p.lr_rot = tc->lr_rotation;
        p.lr_sh = tc->lr_feature;
        p.lr_opac = tc->lr_opacity;
        p.beta1 = tc->adam_beta1;
        p.beta2 = tc->adam_beta2;
        p.eps = tc->adam_eps;
        // optimizer.cpp:75-76 (the step counter was advanced by the caller)
        p.bc1 = 1.0f / (1.0f - std::pow(tc->adam_beta1, (float)c->adam_step));
        p.bc2 = 1.0f / (1.0f - std::pow(tc->adam_beta2, (float)c->adam_step));
    }
}

// Fills the next pinned parameter slot and queues its copy to the device.
int push_params(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg, const gs3d_train_config* tc,
                int iteration, const float* gt_dev, const float* raw_rot_dev = nullptr) {
    const int slot = c->sp_slot;
    c->sp_slot = (c->sp_slot + 1) % kParamSlots;
    CK(cudaEventSynchronize(c->sp_event[slot]));  // the slot's previous copy has been consumed
    StepParams& p = c->sp_ring[slot];
    fill_params(c, p, cam, cfg, tc, iteration, gt_dev, raw_rot_dev);
    CK(cudaMemcpyAsync(c->sp_dev, &p, sizeof(StepParams), cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->sp_event[slot], c->stream));
    return GS3DC_OK;
}

// Reads the control block back and turns device status bits into a status.
int read_control(gs3dc_ctx* c) {
    CK(cudaMemcpyAsync(c->ctrl_host, c->ctrl, kControlReadback, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->persist_host, c->persist, sizeof(Persist), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->last_pairs = c->ctrl_host->total_pairs;
    if (c->ctrl_host->status & kStatusTimeout)
        return fail(c, GS3DC_ERR_DEVICE_TIMEOUT, "a device-side wait exceeded %u polls", c->spin_limit);
    return GS3DC_OK;
}

// ---- autotuner ----

// The pixels per thread of this step: the tuned values, or the next
// candidate while the workload shape is being tuned (returns true then).
bool tune_begin(gs3dc_ctx* c, gs3dc_ctx::Tune& t, const long long key[6]) {
    c->fwd_batch = c->bwd_batch = 128;
    if (c->forced_ppt) {
        c->fwd_ppt = c->bwd_ppt = c->forced_ppt;
        if (c->forced_batch) c->fwd_batch = c->bwd_batch = c->forced_batch;
        return false;
    }
    if (!c->autotune) {
        c->fwd_ppt = c->bwd_ppt = 2;
        return false;
    }
    if (std::memcmp(t.key, key, sizeof(t.key)) != 0) {
        t = gs3dc_ctx::Tune();
        std::memcpy(t.key, key, sizeof(t.key));
    }
    if (t.done) {
        c->fwd_ppt = t.fwd_ppt;
        c->bwd_ppt = t.bwd_ppt;
        c->fwd_batch = t.fwd_batch;
        c->bwd_batch = t.bwd_batch;
        return false;
    }
    if (t.trial < kTunePptSteps) {
        c->fwd_ppt = c->bwd_ppt = kTunePpt[t.trial / kTuneReps];
    } else {
        c->fwd_ppt = t.fwd_ppt;
        c->bwd_ppt = t.bwd_ppt;
        c->fwd_batch = c->bwd_batch = kTuneBatch[(t.trial - kTunePptSteps) / kTuneReps];
    }
    return true;
}

// Adds a trial's rasteriser times; after the pixels-per-thread trials keeps the
// fastest of those, after the batch trials the fastest batch.
void tune_end(gs3dc_ctx* c, gs3dc_ctx::Tune& t, float fwd_ms, float bwd_ms) {
    if (t.trial < kTunePptSteps) {
        const int k = t.trial / kTuneReps;
        t.fwd_ms[k] += fwd_ms;
        t.bwd_ms[k] += bwd_ms;
    } else {
        const int k = (t.trial - kTunePptSteps) / kTuneReps;
        t.fwd_bms[k] += fwd_ms;
        t.bwd_bms[k] += bwd_ms;
    }
    ++t.trial;
    if (t.trial == kTunePptSteps) {
        int bf = 0, bb = 0;
        for (int i = 1; i < 3; i++) {
            if (t.fwd_ms[i] < t.fwd_ms[bf]) bf = i;
            if (t.bwd_ms[i] < t.bwd_ms[bb]) bb = i;
        }
        t.fwd_ppt = kTunePpt[bf];
        t.bwd_ppt = kTunePpt[bb];
        return;
    }
    if (t.trial < kTuneSteps) return;
    // batch 128 at the picked pixels per thread against 64 and 256 (same number of timed steps each)
    float best_f = t.fwd_ms[t.fwd_ppt == 1 ? 0 : t.fwd_ppt == 2 ? 1 : 2];
    float best_b = t.bwd_ms[t.bwd_ppt == 1 ? 0 : t.bwd_ppt == 2 ? 1 : 2];
    for (int i = 0; i < 2; i++) {
        if (t.fwd_bms[i] < best_f) {
            best_f = t.fwd_bms[i];
            t.fwd_batch = kTuneBatch[i];
        }
        if (t.bwd_bms[i] < best_b) {
            best_b = t.bwd_bms[i];
            t.bwd_batch = kTuneBatch[i];
        }
    }
    t.done = true;   // graph keys hold the settings: the next step captures the chosen kernels
    (void)c;
}

// The tuning state of a single-view workload shape (least recently used replaced).
gs3dc_ctx::Tune& tune_slot(gs3dc_ctx* c, const long long key[6]) {
    gs3dc_ctx::Tune* v = &c->tune_single[0];
    for (auto& t : c->tune_single) {
        if (std::memcmp(t.key, key, sizeof(t.key)) == 0) {
            t.used = ++c->tclock;
            return t;
        }
        if (t.used < v->used) v = &t;
    }
    *v = gs3dc_ctx::Tune();
    std::memcpy(v->key, key, sizeof(v->key));
    v->used = ++c->tclock;
    return *v;
}

// ---- launch sequences ----

size_t ctrl_bytes_for(int N) {
    return ((sizeof(Control) + 255) / 256) * 256 + (((size_t)N + kBlock - 1) / kBlock) * sizeof(unsigned long long);
}

// Records the start of `stage` when stage timing is on (un-captured runs only).
int mark(gs3dc_ctx* c, int stage) {
    if (c->stage_timing) CK(cudaEventRecord(c->stage_ev[stage], c->stream));
    return GS3DC_OK;
}

int seq_preprocess(gs3dc_ctx* c, bool cache) {
    int rc = mark(c, GS3DC_STAGE_MEMSETS);
    if (rc) return rc;
    CK(cudaMemsetAsync(c->ctrl_region.p, 0, ctrl_bytes_for(c->N), c->stream));
    CK(cudaMemsetAsync(c->ranges.p, 0, 2 * (size_t)c->num_tiles * sizeof(unsigned), c->stream));
    if ((rc = mark(c, GS3DC_STAGE_PREPROCESS))) return rc;
    PairPtrs pr{c->keys[0].p, c->vals[0].p, c->cap, c->scan_desc};
    if (c->mode_e3) {
        CK(launch_e3_view(c->stream, c->sp_dev, c->num_tiles, e3_ptrs(c)));
        CK(launch_preprocess_e3(c->stream, c->sp_dev, c->N, c->model_raw, model_ptrs(c),
                                c->have_filt3d && !c->model_raw ? c->filt3d.p : nullptr, screen_ptrs(c, false),
                                e3_ptrs(c), pr, c->ctrl));
        c->kernels_last += 1 + (c->N > 0 ? 1 : 0);
        return GS3DC_OK;
    }
    CK(launch_preprocess_plain(c->stream, c->sp_dev, c->N, c->model_raw, cache, model_ptrs(c),
                               screen_ptrs(c, cache), pr, c->ctrl));
    c->kernels_last += c->N > 0 ? 1 : 0;
    return GS3DC_OK;
}

// Sort scratch zeroing; seq_preprocess already did it for a full step.
int seq_sort_scratch(gs3dc_ctx* c) {
    CK(cudaMemsetAsync(&c->ctrl->tickets[1], 0, sizeof(Control) - offsetof(Control, tickets) - sizeof(unsigned),
                       c->stream));
    CK(cudaMemsetAsync(c->ranges.p, 0, 2 * (size_t)c->num_tiles * sizeof(unsigned), c->stream));
    return GS3DC_OK;
}

int seq_sort(gs3dc_ctx* c) {
    CK(cudaMemsetAsync(c->sort_desc.p, 0, (size_t)c->sort_passes * c->sort_desc_stride * sizeof(unsigned long long),
                       c->stream));
    int rc = mark(c, GS3DC_STAGE_SORT_HIST);
    if (rc) return rc;
    int which = 0;
    CK(launch_radix_sort(c->stream, c->sp_dev, c->sort_passes, c->cap, c->keys[0].p, c->vals[0].p, c->keys[1].p,
                         c->vals[1].p, c->sort_desc.p, c->sort_desc_stride, c->ctrl, &which,
                         c->stage_timing ? c->stage_ev[GS3DC_STAGE_SORT_PASSES] : nullptr));
    c->sorted_which = which;
    if ((rc = mark(c, GS3DC_STAGE_RANGES))) return rc;
    CK(launch_tile_ranges(c->stream, c->cap, c->keys[which].p, c->ranges.p, c->ctrl));
    CK(launch_tile_order(c->stream, c->ranges.p, c->num_tiles, c->tile_order.p));
    c->kernels_last += 3 + c->sort_passes;
    return GS3DC_OK;
}


int ensure_depth_sort(gs3dc_ctx* c) {
    const size_t n = c->N > 0 ? (size_t)c->N : 1;
    for (int b = 0; b < 2; b++) {
        CK(c->dkeys[b].ensure(n));
        CK(c->dvals[b].ensure(n));
    }
    c->ddesc_stride = ((n + kSortTile - 1) / kSortTile) * 256ull;
    CK(c->ddesc.ensure(kDepthDigits * c->ddesc_stride));
    CK(c->c_rects.ensure(n));   // tile rectangles for the pair emission (both forms)
    return GS3DC_OK;
}

// Depth-first front half of a train step: preprocess without emission, stable
// depth sort of the Gaussians, pair emission in depth order, stable sort of
// the pairs on the tile bits only (passes kDepthDigits..sort_passes-1 of the
// full key), tile ranges and order.
int seq_front_depth_first(gs3dc_ctx* c) {
    int rc = mark(c, GS3DC_STAGE_MEMSETS);
    if (rc) return rc;
    const int tile_digits = c->sort_passes - kDepthDigits;
    {
        // control block, tile ranges and both look-back descriptor sets, in one launch
        ClearRegions z{};
        z.p[0] = reinterpret_cast<unsigned long long*>(c->ctrl_region.p);
        z.words[0] = ctrl_bytes_for(c->N) / 8;
        z.p[1] = reinterpret_cast<unsigned long long*>(c->ranges.p);
        z.words[1] = (size_t)c->num_tiles;   // 2 u32 per tile
        z.p[2] = c->ddesc.p;
        z.words[2] = kDepthDigits * c->ddesc_stride;
        z.p[3] = tile_digits > 0 ? c->sort_desc.p : nullptr;
        z.words[3] = tile_digits > 0 ? (size_t)tile_digits * c->sort_desc_stride : 0;
        CK(launch_clear_regions(c->stream, z));
    }
    if ((rc = mark(c, GS3DC_STAGE_PREPROCESS))) return rc;
    // tile-only keys live in the (otherwise unused) 64-bit key buffers
    unsigned* tk[2] = {reinterpret_cast<unsigned*>(c->keys[0].p), reinterpret_cast<unsigned*>(c->keys[1].p)};
    PairPtrs pr{c->keys[0].p, c->vals[0].p, c->cap, c->scan_desc, tk[0]};
    const bool chosen = chosen_form(c);
    if (chosen)
        CK(launch_chosen_preprocess(c->stream, c->sp_dev, c->N, c->form == GS3DC_FORM_FP16, chosen_ptrs(c),
                                    screen_ptrs(c, false), DepthKeys{c->dkeys[0].p, c->dvals[0].p}, c->c_rects.p,
                                    c->ctrl));
    else
        CK(launch_preprocess_plain(c->stream, c->sp_dev, c->N, c->model_raw, false, model_ptrs(c),
                                   screen_ptrs(c, false), pr, c->ctrl,
                                   DepthKeys{c->dkeys[0].p, c->dvals[0].p, false, c->c_rects.p}));
    if ((rc = mark(c, GS3DC_STAGE_SORT_HIST))) return rc;
    // the reduced form orders by the depth's upper 24 bits (relative steps of 2^-15; ties keep index order)
    const int depth_first_digit = chosen ? kChosenDepthSkip : 0;
    int dw = 0;
    CK(launch_radix_sort32(c->stream, c->sp_dev, kDepthDigits, 0, false, (unsigned long long)c->N, c->dkeys[0].p,
                           c->dvals[0].p, c->dkeys[1].p, c->dvals[1].p, c->ddesc.p, c->ddesc_stride, c->ctrl, &dw,
                           nullptr, &c->ctrl->gauss_keys, depth_first_digit));
    CK(launch_emit_ranked(c->stream, c->sp_dev, c->N, c->dvals[dw].p, screen_ptrs(c, false), pr, c->ctrl,
                          c->c_rects.p));
    if ((rc = mark(c, GS3DC_STAGE_SORT_PASSES))) return rc;
    int which = 0;
    CK(launch_radix_sort32(c->stream, c->sp_dev, tile_digits, kDepthDigits, true, c->cap, tk[0], c->vals[0].p, tk[1],
                           c->vals[1].p, c->sort_desc.p, c->sort_desc_stride, c->ctrl, &which));
    c->sorted_which = which;
    if ((rc = mark(c, GS3DC_STAGE_RANGES))) return rc;
    CK(launch_tile_ranges32(c->stream, c->cap, tk[which], c->ranges.p, c->ctrl));
    CK(launch_tile_order(c->stream, c->ranges.p, c->num_tiles, c->tile_order.p));
    // clearing, preprocess, depth histogram + passes, emission, tile passes, ranges + order
    c->kernels_last +=
        1 + (c->N > 0 ? 1 + (1 + kDepthDigits - depth_first_digit) + 1 + (tile_digits > 0 ? tile_digits : 0) + 2 : 2);
    return GS3DC_OK;
}

// Back half of a train step of the reduced-storage form: fast-exp
// rasterisers, fused adjoint + Adam.
// The train step's forward rasteriser: with the fused L1, or (loss_later: the
// target is still being copied in) without the loss.
int seq_train_forward(gs3dc_ctx* c, bool loss_later) {
    const int w = c->sorted_which;
    if (chosen_form(c))
        CK(launch_raster_fwd_fast(c->stream, c->sp_dev, c->num_tiles, c->ranges.p, c->tile_order.p, c->vals[w].p,
                                  screen_ptrs(c, false), pixel_ptrs(c), c->ctrl, c->fwd_ppt, c->fwd_batch, loss_later));
    else
        CK(launch_raster_fwd_plain(c->stream, c->sp_dev, c->num_tiles, true, c->ranges.p, c->tile_order.p,
                                   c->vals[w].p, screen_ptrs(c, false), pixel_ptrs(c), c->ctrl, c->fwd_ppt,
                                   c->fwd_batch, loss_later));
    return GS3DC_OK;
}

int seq_back_chosen(gs3dc_ctx* c, bool loss_later) {
    int rc;
    const int w = c->sorted_which;
    if (loss_later) {
        CK(launch_l1_loss(c->stream, c->sp_dev, pixel_ptrs(c), (size_t)c->W * c->H, c->ctrl));
        c->kernels_last += 1;
    } else {
        if ((rc = mark(c, GS3DC_STAGE_RASTER_FWD))) return rc;
        if ((rc = seq_train_forward(c, false))) return rc;
    }
    if ((rc = mark(c, GS3DC_STAGE_RASTER_BWD))) return rc;
    CK(launch_raster_bwd_fast(c->stream, c->sp_dev, c->num_tiles, c->ranges.p, c->tile_order.p, c->vals[w].p,
                              screen_ptrs(c, false), pixel_ptrs(c), rgrad_ptrs(c), c->ctrl, c->bwd_ppt,
                              c->bwd_batch));
    if ((rc = mark(c, GS3DC_STAGE_PREPROCESS_BWD))) return rc;
    CK(launch_chosen_backward_adam(c->stream, c->sp_dev, c->N, c->max_coeffs * 3, c->form == GS3DC_FORM_FP16,
                                   chosen_ptrs(c), rgrad_ptrs(c),
                                   c->keep_grads ? grad_ptrs(c) : GradPtrs{nullptr, nullptr, nullptr, nullptr, nullptr},
                                   c->ctrl));
    if ((rc = mark(c, GS3DC_NUM_STAGES))) return rc;
    c->kernels_last += 3;
    return GS3DC_OK;
}

// Front half of a train step: preprocess, pair emission, sort, tile ranges
// (loss_later: and the forward rasteriser without the loss, which then
// overlaps the target's copy too).
int seq_train_front(gs3dc_ctx* c, bool loss_later = false) {
    int rc;
    c->mode_e3 = false;   // training is the 2D path only
    c->screen_n = c->N;
    c->screen_imported = false;
    if (chosen_form(c) || c->sort_mode == GS3DC_SORT_DEPTH_FIRST) {
        if ((rc = seq_front_depth_first(c))) return rc;
    } else {
        if ((rc = seq_preprocess(c, false))) return rc;
        if ((rc = seq_sort(c))) return rc;
    }
    if (loss_later) {
        if ((rc = mark(c, GS3DC_STAGE_RASTER_FWD))) return rc;
        if ((rc = seq_train_forward(c, true))) return rc;
    }
    return GS3DC_OK;
}

// Back half: forward rasteriser with the fused L1 (the only reader of the
// target) or, after a loss_later front half, the L1 alone; backward
// rasteriser, preprocess backward, optimiser.
int seq_train_back(gs3dc_ctx* c, bool loss_later = false) {
    int rc;
    if (chosen_form(c)) return seq_back_chosen(c, loss_later);
    const int w = c->sorted_which;
    if (loss_later) {
        CK(launch_l1_loss(c->stream, c->sp_dev, pixel_ptrs(c), (size_t)c->W * c->H, c->ctrl));
        c->kernels_last += 1;
    } else {
        if ((rc = mark(c, GS3DC_STAGE_RASTER_FWD))) return rc;
        if ((rc = seq_train_forward(c, false))) return rc;
    }
    if ((rc = mark(c, GS3DC_STAGE_RASTER_BWD))) return rc;
    CK(launch_raster_bwd_plain(c->stream, c->sp_dev, c->num_tiles, true, c->ranges.p, c->tile_order.p, c->vals[w].p,
                               screen_ptrs(c, false), pixel_ptrs(c), rgrad_ptrs(c), c->ctrl, c->bwd_ppt,
                              c->bwd_batch));
    if ((rc = mark(c, GS3DC_STAGE_PREPROCESS_BWD))) return rc;
    if (c->fused_adam && !c->keep_grads) {
        CK(launch_preprocess_bwd_plain(c->stream, c->sp_dev, c->N, c->max_coeffs * 3, 1, model_ptrs(c),
                                       adam_ptrs(c), screen_ptrs(c, false), rgrad_ptrs(c), grad_ptrs(c), c->ctrl));
    } else {
        CK(launch_preprocess_bwd_plain(c->stream, c->sp_dev, c->N, c->max_coeffs * 3, 2, model_ptrs(c),
                                       adam_ptrs(c), screen_ptrs(c, false), rgrad_ptrs(c), grad_ptrs(c), c->ctrl));
        CK(launch_optimizer_plain(c->stream, c->sp_dev, c->N, c->max_coeffs * 3, model_ptrs(c), adam_ptrs(c),
                                  grad_ptrs(c), c->ctrl));
        c->kernels_last += 1;
    }
    if ((rc = mark(c, GS3DC_NUM_STAGES))) return rc;
    c->kernels_last += 3;
    return GS3DC_OK;
}

int require_model(gs3dc_ctx* c) {
    if (!c->have_model) return fail(c, GS3DC_ERR_NO_MODEL, "no model uploaded");
    return GS3DC_OK;
}

// Runs the preprocess, growing the pair capacity once if it overflowed.
int run_preprocess(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg, bool cache) {
    int rc = ensure_pixels(c, cam->width, cam->height);
    if (rc) return rc;
    // the 3D mode keeps no 2D ForwardCache (preprocessor_cpu.cpp:36)
    c->mode_e3 = cfg->eval_3D;
    if (c->mode_e3) {
        cache = false;
        if ((rc = ensure_e3(c, c->N))) return rc;
    }
    if (c->cap == 0 || c->sort_num_tiles != c->num_tiles) {
        unsigned long long guess = c->min_cap ? c->min_cap : (unsigned long long)c->N * 8ull;
        rc = ensure_pairs(c, guess > c->cap ? guess : c->cap, c->num_tiles);
        if (rc) return rc;
    }
    if (cache && (rc = ensure_cache(c))) return rc;
    for (int attempt = 0; attempt < 2; attempt++) {
        c->kernels_last = 0;
        rc = push_params(c, cam, cfg, nullptr, 0, nullptr);
        if (rc) return rc;
        rc = seq_preprocess(c, cache);
        if (rc) return rc;
        rc = read_control(c);
        if (rc) return rc;
        if (c->last_pairs <= c->cap) break;
        rc = ensure_pairs(c, c->last_pairs + c->last_pairs / 4 + 4096, c->num_tiles);
        if (rc) return rc;
    }
    c->have_screen = true;
    c->have_pairs = true;
    c->have_sorted = c->have_raster = c->have_rgrad = false;
    c->screen_n = c->N;
    c->screen_imported = false;
    return GS3DC_OK;
}

int download(gs3dc_ctx* c, void* host, const void* dev, size_t bytes) {
    if (!host || bytes == 0) return GS3DC_OK;
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    return GS3DC_OK;
}

int upload_model_arrays(gs3dc_ctx* c, int N, int sh_degree, int mc, const float* p, const float* s, const float* r,
                        const float* sh, const float* o) {
    if (N < 0 || mc <= 0 || mc > 16 || sh_degree < 0 || sh_degree > 3 || (sh_degree + 1) * (sh_degree + 1) > mc)
        return fail(c, GS3DC_ERR_INVALID_ARG, "bad model shape N=%d sh_degree=%d max_coeffs=%d", N, sh_degree, mc);
    if (N > 0 && (!p || !s || !r || !sh || !o)) return fail(c, GS3DC_ERR_INVALID_ARG, "model arrays must be non-NULL");
    if (c->N != N || c->max_coeffs != mc) drop_graphs(c);
    int rc = ensure_model(c, N, mc);
    if (rc) return rc;
    c->N = N;
    c->sh_degree = sh_degree;
    c->max_coeffs = mc;
    const size_t n = (size_t)N;
    if (N > 0) {
        CK(cudaMemcpyAsync(c->pos.p, p, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->sc.p, s, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->rot.p, r, 4 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->sh.p, sh, 3 * n * mc * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->op.p, o, n * 4, cudaMemcpyHostToDevice, c->stream));
        // raster-gradient accumulators start at zero (the fused step re-zeroes them)
        CK(cudaMemsetAsync(c->dm2.p, 0, 2 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->dcon.p, 0, 3 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->drgb.p, 0, 3 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->dop.p, 0, n * 4, c->stream));
    }
    c->have_model = true;
    c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
    return GS3DC_OK;
}

// ---- checkpoint / resume ----

constexpr char kCkptMagic[8] = {'G', 'S', '3', 'D', 'C', 'K', 'P', 'T'};
constexpr uint32_t kCkptVersion = 1;

struct CkptHeader {
    char magic[8];
    uint32_t version;
    int32_t form, count, sh_degree, max_coeffs, adam_step;
    int32_t reserved[4];
};

// The byte sizes of a form's arrays, in file order.
std::vector<size_t> state_sizes(int form, size_t n, size_t mc3) {
    if (form != GS3DC_FORM_PLAIN_FP32)   // 16-bit model, BF16 moments, FP32 positions and their moments
        return {12 * n, 16 * n, 2 * mc3 * n, 12 * n, 12 * n, 16 * n, 16 * n, 2 * mc3 * n, 2 * mc3 * n};
    return {12 * n, 12 * n, 16 * n, 4 * mc3 * n, 4 * n,                 // positions, scales, rotations, SH, opacity
            12 * n, 12 * n, 12 * n, 12 * n, 16 * n, 16 * n,             // their first / second moments
            4 * mc3 * n, 4 * mc3 * n, 4 * n, 4 * n};
}

// The device arrays of the current form, in file order.
std::vector<void*> state_arrays(gs3dc_ctx* c) {
    if (chosen_form(c))
        return {c->c_pos.p, c->c_attr.p, c->c_sh.p, c->cm_pos.p, c->cv_pos.p,
                c->cm_attr.p, c->cv_attr.p, c->cm_sh.p, c->cv_sh.p};
    return {c->pos.p, c->sc.p, c->rot.p, c->sh.p, c->op.p, c->m_pos.p, c->v_pos.p, c->m_sc.p,
            c->v_sc.p, c->m_rot.p, c->v_rot.p, c->m_sh.p, c->v_sh.p, c->m_op.p, c->v_op.p};
}

// ---- multi-view train step ----

struct BatchShape {
    int V = 0;
    long long VN = 0;
    long long seg = 0;         // each view's depth-sort segment: N rounded up to whole 8192-key sort tiles
    long long VS = 0;          // V * seg: depth-sort keys (the emission's ranks)
    unsigned tiles = 0;        // all views' tiles
    unsigned long long pix = 0;  // all views' pixels
    int tile_digits = 0;
};

ScreenPtrs batch_screen(gs3dc_ctx* c) {
    auto& b = c->batch;
    // the reduced form keeps no depth, radius or tile-count arrays (the rectangles stand for them)
    return {b.rec0.p, b.rec1.p, b.cbt.p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
}
PixelPtrs batch_pixels(gs3dc_ctx* c) {
    auto& b = c->batch;
    return {b.image.p, b.T.p, nullptr, b.last.p, b.dsign.p, nullptr};
}
RGradPtrs batch_rgrads(gs3dc_ctx* c) {
    auto& b = c->batch;
    return {b.dm2.p, b.dcon.p, b.drgb.p, b.dop.p};
}

// Pair buffers and tile-sort descriptors of the multi-view step.
int batch_pairs(gs3dc_ctx* c, unsigned long long cap, int digits) {
    auto& b = c->batch;
    if (cap > 0xFFFFFFFFull)
        return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "%llu tile pairs exceed the 32-bit tile-range format", cap);
    if (cap > b.cap) {
        for (int k = 0; k < 2; k++) {
            CK(b.keys[k].ensure(cap));
            CK(b.vals[k].ensure(cap));
        }
        b.cap = cap;
    }
    const unsigned long long stride = ((b.cap + kSortTile - 1) / kSortTile) * 256ull;
    CK(b.sort_desc.ensure((size_t)(digits > 1 ? digits : 1) * stride));
    return GS3DC_OK;
}

// Buffers of a multi-view step with the given shape.
int batch_buffers(gs3dc_ctx* c, const BatchShape& sh) {
    auto& b = c->batch;
    const size_t vn = (size_t)sh.VN;
    CK(b.views.ensure((size_t)sh.V));
    CK(b.rec0.ensure(vn));
    CK(b.rec1.ensure(vn));
    CK(b.cbt.ensure(vn));
    CK(b.rects.ensure(vn));
    if (b.dm2.n < 2 * vn) b.grads_zeroed = 0;
    CK(b.dm2.ensure(2 * vn));
    CK(b.dcon.ensure(3 * vn));
    CK(b.drgb.ensure(3 * vn));
    CK(b.dop.ensure(vn));
    if (b.grads_zeroed < vn) {
        // the accumulators start at zero; the backward re-zeroes what it reads
        CK(cudaMemsetAsync(b.dm2.p, 0, b.dm2.n * 4, c->stream));
        CK(cudaMemsetAsync(b.dcon.p, 0, b.dcon.n * 4, c->stream));
        CK(cudaMemsetAsync(b.drgb.p, 0, b.drgb.n * 4, c->stream));
        CK(cudaMemsetAsync(b.dop.p, 0, b.dop.n * 4, c->stream));
        b.grads_zeroed = b.dop.n;
    }
    const size_t vs = (size_t)sh.VS;   // the depth sort's padded per-view segments
    for (int k = 0; k < 2; k++) {
        CK(b.dkeys[k].ensure(vs));
        CK(b.dvals[k].ensure(vs));
    }
    CK(b.ddesc.ensure(3 * ((vs + kSortTile - 1) / kSortTile) * 256));
    CK(b.seg_hist.ensure((size_t)sh.V * 3 * 256));
    CK(b.image.ensure(3 * sh.pix));
    CK(b.T.ensure(sh.pix));
    CK(b.last.ensure(sh.pix));
    CK(b.dsign.ensure(sh.pix));
    CK(b.ranges.ensure(2 * (size_t)sh.tiles));
    CK(b.order.ensure(sh.tiles));
    CK(b.hist_parts.ensure((size_t)kHistParts * (kMaxPasses - kDepthDigits) * 256));
    Control* before = c->ctrl;
    int rc = ensure_ctrl(c, (int)std::min<long long>(sh.VS, 0x7fffffffLL));
    if (rc) return rc;
    if (c->ctrl != before) drop_graphs(c);   // captured launches hold the control block's address
    return GS3DC_OK;
}

// One multi-view step: preprocess of every (view, Gaussian), stable sort by
// (view, depth's upper 24 bits) in 4 passes, emission in that order with global tile ids,
// stable sort of the pairs on the tile bits, ranges and a heavy-first order of
// all views' tiles, persistent forward and backward rasterisers over that
// order, then the adjoint summed over the views and one Adam step.
int seq_batch(gs3dc_ctx* c, const BatchShape& sh) {
    auto& b = c->batch;
    const StepParams* views = b.views.p;
    const unsigned long long vs = (unsigned long long)sh.VS;
    const unsigned long long dstride = ((vs + kSortTile - 1) / kSortTile) * 256ull;
    const unsigned long long pstride = ((b.cap + kSortTile - 1) / kSortTile) * 256ull;
    CK(cudaMemsetAsync(c->ctrl_region.p, 0, ctrl_bytes_for((int)std::min<long long>(sh.VS, 0x7fffffffLL)),
                       c->stream));
    CK(cudaMemsetAsync(b.ranges.p, 0, 2 * (size_t)sh.tiles * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(b.ddesc.p, 0, 3 * dstride * sizeof(unsigned long long), c->stream));
    CK(cudaMemsetAsync(b.seg_hist.p, 0, (size_t)sh.V * 3 * 256 * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(b.hist_parts.p, 0, b.hist_parts.n * sizeof(unsigned), c->stream));
    if (sh.tile_digits > 0)
        CK(cudaMemsetAsync(b.sort_desc.p, 0, (size_t)sh.tile_digits * pstride * sizeof(unsigned long long),
                           c->stream));
    DepthKeys dk{b.dkeys[0].p, b.dvals[0].p};
    dk.views24 = true;
    dk.seg_keys = (unsigned long long)sh.seg;
    CK(launch_chosen_preprocess(c->stream, views, c->N, c->form == GS3DC_FORM_FP16, chosen_ptrs(c), batch_screen(c),
                                dk, b.rects.p, c->ctrl, sh.V));
    // 32-bit keys (view << 24 | the depth's upper 24 bits), view v's in segment v (entries already
    // grouped by view): each segment sorted apart on the three depth digits
    int dw = 0;
    CK(launch_radix_sort32_segmented(c->stream, views, 0, 3, vs, (unsigned long long)sh.seg, b.dkeys[0].p,
                                     b.dvals[0].p, b.dkeys[1].p, b.dvals[1].p, b.ddesc.p, dstride, b.seg_hist.p,
                                     c->ctrl, &dw));
    PairPtrs pr{nullptr, b.vals[0].p, b.cap, c->scan_desc, b.keys[0].p};
    CK(launch_emit_ranked(c->stream, views, (int)vs, b.dvals[dw].p, batch_screen(c), pr, c->ctrl, b.rects.p, c->N,
                          5, b.hist_parts.p));
    int which = 0;
    CK(launch_radix_sort32(c->stream, views, sh.tile_digits, 5, true, b.cap, b.keys[0].p, b.vals[0].p, b.keys[1].p,
                           b.vals[1].p, b.sort_desc.p, pstride, c->ctrl, &which));
    CK(launch_tile_ranges_views(c->stream, b.cap, b.keys[which].p, views, b.ranges.p, c->ctrl));
    CK(launch_tile_order(c->stream, b.ranges.p, (int)sh.tiles, b.order.p, c->ctrl));
    const bool tuning = c->autotune && !c->tune_batch.done;
    if (tuning) CK(cudaEventRecord(c->tune_ev[0], c->stream));
    CK(launch_raster_fwd_fast_multi(c->stream, views, sh.V, sh.tiles, b.ranges.p, b.order.p, b.vals[which].p,
                                    batch_screen(c), batch_pixels(c), c->ctrl, c->fwd_ppt, c->fwd_batch));
    if (tuning) CK(cudaEventRecord(c->tune_ev[1], c->stream));
    CK(launch_raster_bwd_fast_multi(c->stream, views, sh.V, sh.tiles, b.ranges.p, b.order.p, b.vals[which].p,
                                    batch_screen(c), batch_pixels(c), batch_rgrads(c), c->ctrl, c->bwd_ppt,
                                    c->bwd_batch));
    if (tuning) CK(cudaEventRecord(c->tune_ev[2], c->stream));
    CK(launch_chosen_backward_adam(c->stream, views, c->N, c->max_coeffs * 3, c->form == GS3DC_FORM_FP16,
                                   chosen_ptrs(c), batch_rgrads(c),
                                   c->keep_grads ? grad_ptrs(c) : GradPtrs{nullptr, nullptr, nullptr, nullptr, nullptr},
                                   c->ctrl, sh.V));
    // preprocess, 4 depth passes, emission + its count reduction, tile passes, ranges + order, rasterisers,
    // adjoint
    c->kernels_last = 1 + 4 + 2 + (sh.tile_digits > 0 ? sh.tile_digits : 0) + 1 + (sh.tiles > 65536 ? 2 : 1) + 3;
    return GS3DC_OK;
}

}  // namespace

// ======================================================================
extern "C" {

const char* gs3dc_status_string(int s) {
    switch (s) {
        case GS3DC_OK: return "ok";
        case GS3DC_ERR_INVALID_ARG: return "invalid argument";
        case GS3DC_ERR_CUDA: return "CUDA error";
        case GS3DC_ERR_PAIR_OVERFLOW: return "tile-pair capacity overflow";
        case GS3DC_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case GS3DC_ERR_NO_MODEL: return "no model uploaded";
        case GS3DC_ERR_OUT_OF_MEMORY: return "out of device memory";
        case GS3DC_ERR_STATE: return "stage called out of order";
        default: return "unknown status";
    }
}

const char* gs3dc_last_error(const gs3dc_ctx* c) { return c ? c->err.c_str() : "null context"; }

int gs3dc_create(int device, gs3dc_ctx** out) {
    if (!out) return GS3DC_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return GS3DC_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return GS3DC_ERR_CUDA;
    if (prop.major != 10) return GS3DC_ERR_CUDA;  // built for sm_100a only; no fallback path exists
    gs3dc_ctx* c = new gs3dc_ctx();
    c->device = device;
    auto bail = [&](int code) {
        gs3dc_destroy(c);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    if (cudaEventCreateWithFlags(&c->ev_gt_ready, cudaEventDisableTiming) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    for (int k = 0; k < 3; k++)
        if (cudaEventCreate(&c->tune_ev[k]) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    for (int b = 0; b < 2; b++)
        if (cudaEventCreateWithFlags(&c->ev_gt_free[b], cudaEventDisableTiming) != cudaSuccess)
            return bail(GS3DC_ERR_CUDA);
    if (cudaMalloc(&c->sp_dev, sizeof(StepParams)) != cudaSuccess) return bail(GS3DC_ERR_OUT_OF_MEMORY);
    if (cudaMalloc(&c->persist, sizeof(Persist)) != cudaSuccess) return bail(GS3DC_ERR_OUT_OF_MEMORY);
    if (cudaMemset(c->persist, 0, sizeof(Persist)) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    if (cudaMallocHost(&c->persist_host, sizeof(Persist)) != cudaSuccess) return bail(GS3DC_ERR_OUT_OF_MEMORY);
    std::memset(c->persist_host, 0, sizeof(Persist));
    if (cudaMallocHost(&c->sp_ring, kParamSlots * sizeof(StepParams)) != cudaSuccess) return bail(GS3DC_ERR_OUT_OF_MEMORY);
    if (cudaMallocHost(&c->ctrl_host, sizeof(Control)) != cudaSuccess) return bail(GS3DC_ERR_OUT_OF_MEMORY);
    for (int k = 0; k < kParamSlots; k++)
        if (cudaEventCreateWithFlags(&c->sp_event[k], cudaEventDisableTiming) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    for (int k = 0; k <= GS3DC_NUM_STAGES; k++)
        if (cudaEventCreate(&c->stage_ev[k]) != cudaSuccess) return bail(GS3DC_ERR_CUDA);
    if (ensure_model(c, 0, 1) != GS3DC_OK) return bail(GS3DC_ERR_OUT_OF_MEMORY);
    *out = c;
    return GS3DC_OK;
}

void gs3dc_destroy(gs3dc_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    drop_graphs(c);
    DevBuf<float>* fb[] = {&c->pos,    &c->sc,      &c->rot,     &c->sh,     &c->op,      &c->m_pos,  &c->v_pos,
                           &c->m_sc,   &c->v_sc,    &c->m_rot,   &c->v_rot,  &c->m_sh,    &c->v_sh,   &c->m_op,
                           &c->v_op,   &c->g_pos,   &c->g_sc,    &c->g_rot,  &c->g_sh,    &c->g_op,
                           &c->depth,  &c->c_cov3D, &c->c_pview, &c->c_phw,  &c->c_cov2D, &c->c_det,  &c->x_means2D,
                           &c->x_depths, &c->x_conics, &c->x_opac, &c->x_rgb, &c->dm2,    &c->dcon,   &c->drgb,
                           &c->dop,    &c->image,   &c->T_final, &c->d_image, &c->gt};
    for (auto* b : fb) b->release();
    c->cbt.release();
    c->rec0.release();
    c->rec1.release();
    c->radius.release();
    c->tiles.release();
    c->x_radii.release();
    c->x_tiles.release();
    c->n_contrib.release();
    for (int b = 0; b < 2; b++) {
        c->keys[b].release();
        c->vals[b].release();
    }
    c->sort_desc.release();
    c->raw_rot_tmp.release();
    c->ctrl_region.release();
    c->ranges.release();
    c->tile_order.release();
    c->last_j.release();
    c->dsign.release();
    if (c->sp_dev) cudaFree(c->sp_dev);
    if (c->persist) cudaFree(c->persist);
    if (c->persist_host) cudaFreeHost(c->persist_host);
    if (c->sp_ring) cudaFreeHost(c->sp_ring);
    if (c->ctrl_host) cudaFreeHost(c->ctrl_host);
    for (int k = 0; k < kParamSlots; k++)
        if (c->sp_event[k]) cudaEventDestroy(c->sp_event[k]);
    for (int k = 0; k <= GS3DC_NUM_STAGES; k++)
        if (c->stage_ev[k]) cudaEventDestroy(c->stage_ev[k]);
    if (c->batch.views_event) cudaEventDestroy(c->batch.views_event);
    if (c->batch.views_host) cudaFreeHost(c->batch.views_host);
    if (c->ev_gt_ready) cudaEventDestroy(c->ev_gt_ready);
    for (int k = 0; k < 3; k++)
        if (c->tune_ev[k]) cudaEventDestroy(c->tune_ev[k]);
    for (int b = 0; b < 2; b++)
        if (c->ev_gt_free[b]) cudaEventDestroy(c->ev_gt_free[b]);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int gs3dc_get_stream(gs3dc_ctx* c, void** stream) {
    if (!c || !stream) return GS3DC_ERR_INVALID_ARG;
    *stream = (void*)c->stream;
    return GS3DC_OK;
}

int gs3dc_set_option(gs3dc_ctx* c, int option, int64_t value) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    switch (option) {
        case GS3DC_OPT_PAIR_CAPACITY:
            if (value < 0) return fail(c, GS3DC_ERR_INVALID_ARG, "negative capacity");
            c->min_cap = (unsigned long long)value;
            return GS3DC_OK;
        case GS3DC_OPT_USE_GRAPH:
            c->use_graph = value != 0;
            return GS3DC_OK;
        case GS3DC_OPT_FORM: {
            if (value != GS3DC_FORM_PLAIN_FP32 && value != GS3DC_FORM_BF16 && value != GS3DC_FORM_FP16)
                return fail(c, GS3DC_ERR_INVALID_ARG, "unknown form %lld", (long long)value);
            if (value == c->form) return GS3DC_OK;
            CK(cudaSetDevice(c->device));
            int rc;
            drop_graphs(c);
            if (c->have_model && !c->model_raw && value != GS3DC_FORM_PLAIN_FP32)
                return fail(c, GS3DC_ERR_STATE, "the device model is an activated render model");
            // the model moves to the new form; the optimiser restarts
            if ((rc = unload_chosen(c))) return rc;
            c->form = (int)value;
            c->chosen_ready = false;
            if (c->have_model && chosen_form(c) && (rc = load_chosen(c))) return rc;
            if (c->have_model && (rc = zero_adam(c))) return rc;
            c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
            CK(cudaStreamSynchronize(c->stream));
            return GS3DC_OK;
        }
        case GS3DC_OPT_DENSITY_SEED:
            c->dc_rng = (unsigned long long)value;
            return GS3DC_OK;
        case GS3DC_OPT_SPIN_LIMIT:
            if (value <= 0) return fail(c, GS3DC_ERR_INVALID_ARG, "spin limit must be positive");
            c->spin_limit = (unsigned)value;
            drop_graphs(c);
            return GS3DC_OK;
        case GS3DC_OPT_FUSED_ADAM:
            c->fused_adam = value != 0;
            return GS3DC_OK;
        case GS3DC_OPT_STAGE_TIMING:
            c->stage_timing = value != 0;
            return GS3DC_OK;
        case GS3DC_OPT_AUTOTUNE:
            c->autotune = value != 0;
            for (auto& t : c->tune_single) t = gs3dc_ctx::Tune();
            c->tune_batch = gs3dc_ctx::Tune();
            drop_graphs(c);
            return GS3DC_OK;
        case GS3DC_OPT_RASTER_PPT:
            if (value != 0 && value != 1 && value != 2 && value != 4)
                return fail(c, GS3DC_ERR_INVALID_ARG, "pixels per thread %lld: 0, 1, 2 or 4", (long long)value);
            c->forced_ppt = (int)value;
            return GS3DC_OK;
        case GS3DC_OPT_RASTER_BATCH:
            if (value != 0 && value != 64 && value != 128 && value != 256)
                return fail(c, GS3DC_ERR_INVALID_ARG, "staging batch %lld: 0, 64, 128 or 256", (long long)value);
            c->forced_batch = (int)value;
            return GS3DC_OK;
        case GS3DC_OPT_KEEP_GRADIENTS:
            c->keep_grads = value != 0;
            drop_graphs(c);
            return GS3DC_OK;
        case GS3DC_OPT_SORT:
            if (value != GS3DC_SORT_DEPTH_FIRST && value != GS3DC_SORT_FULL_KEY)
                return fail(c, GS3DC_ERR_INVALID_ARG, "unknown sort mode %lld", (long long)value);
            c->sort_mode = (int)value;
            return GS3DC_OK;
        default:
            return fail(c, GS3DC_ERR_INVALID_ARG, "unknown option %d", option);
    }
}

int gs3dc_get_stat(gs3dc_ctx* c, int stat, int64_t* value) {
    if (!c || !value) return GS3DC_ERR_INVALID_ARG;
    switch (stat) {
        case GS3DC_STAT_TOTAL_PAIRS: *value = (int64_t)c->last_pairs; return GS3DC_OK;
        case GS3DC_STAT_FWD_PPT: *value = c->fwd_ppt; return GS3DC_OK;
        case GS3DC_STAT_BWD_PPT: *value = c->bwd_ppt; return GS3DC_OK;
        case GS3DC_STAT_FWD_BATCH: *value = c->fwd_batch; return GS3DC_OK;
        case GS3DC_STAT_BWD_BATCH: *value = c->bwd_batch; return GS3DC_OK;
        case GS3DC_STAT_PAIR_CAPACITY: *value = (int64_t)c->cap; return GS3DC_OK;
        case GS3DC_STAT_KERNELS_LAST: *value = c->kernels_last; return GS3DC_OK;
        case GS3DC_STAT_SORT_PASSES: *value = c->sort_passes; return GS3DC_OK;
        case GS3DC_STAT_GRAPH_REPLAYS: *value = c->graph_replays; return GS3DC_OK;
        case GS3DC_STAT_GRAPH_CAPTURES: *value = c->graph_captures; return GS3DC_OK;
        case GS3DC_STAT_ADAM_STEP: *value = c->adam_step; return GS3DC_OK;
        case GS3DC_STAT_NUM_GAUSSIANS: *value = c->N; return GS3DC_OK;
        case GS3DC_STAT_SCREEN_GAUSSIANS: *value = c->screen_n; return GS3DC_OK;
        default: return fail(c, GS3DC_ERR_INVALID_ARG, "unknown stat %d", stat);
    }
}

int gs3dc_set_gaussians(gs3dc_ctx* c, const gs3d_gaussians* g) {
    if (!c || !g) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_set_gaussians")) return rc_;
    CK(cudaSetDevice(c->device));
    int rc = upload_model_arrays(c, g->count, g->sh_degree, g->max_coeffs, g->positions, g->scales, g->rotations,
                                 g->sh_coeffs, g->opacities);
    if (rc) return rc;
    c->model_raw = false;
    // GaussianData::filter_3D (the 3D mode's per-Gaussian mip filter; include/types.h:44)
    c->have_filt3d = g->filter_3D != nullptr && g->count > 0;
    if (c->have_filt3d) {
        CK(c->filt3d.ensure((size_t)g->count));
        CK(cudaMemcpyAsync(c->filt3d.p, g->filter_3D, (size_t)g->count * 4, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_set_raw_params(gs3dc_ctx* c, const gs3d_raw_params* r) {
    if (!c || !r) return GS3DC_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    int rc = upload_model_arrays(c, r->count, r->sh_degree, r->max_coeffs, r->raw_positions, r->raw_scales,
                                 r->raw_rotations, r->raw_sh_coeffs, r->raw_opacities);
    if (rc) return rc;
    c->model_raw = true;
    c->have_filt3d = false;
    c->dc_n = 0;   // a new model: the density statistics restart
    if ((rc = ensure_adam(c))) return rc;
    if ((rc = zero_adam(c))) return rc;
    c->chosen_ready = false;
    if (chosen_form(c) && (rc = load_chosen(c))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_update_raw_params(gs3dc_ctx* c, const gs3d_raw_params* r) {
    if (!c || !r) return GS3DC_ERR_INVALID_ARG;
    int rc = require_model(c);
    if (rc) return rc;
    if (!c->model_raw) return fail(c, GS3DC_ERR_STATE, "the device model is an activated render model");
    if (r->count != c->N || r->max_coeffs != c->max_coeffs || r->sh_degree != c->sh_degree)
        return fail(c, GS3DC_ERR_INVALID_ARG, "update needs the uploaded shape (N=%d, mc=%d)", c->N, c->max_coeffs);
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->N;
    if (n) {
        CK(cudaMemcpyAsync(c->pos.p, r->raw_positions, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->sc.p, r->raw_scales, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->rot.p, r->raw_rotations, 4 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->sh.p, r->raw_sh_coeffs, 3 * n * c->max_coeffs * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->op.p, r->raw_opacities, n * 4, cudaMemcpyHostToDevice, c->stream));
        if (chosen_form(c))
            CK(launch_chosen_from_raw(c->stream, c->N, c->max_coeffs * 3, c->form == GS3DC_FORM_FP16,
                                      ModelPtrs{c->pos.p, c->sc.p, c->rot.p, c->sh.p, c->op.p}, chosen_ptrs(c)));
    }
    CK(cudaStreamSynchronize(c->stream));
    c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
    return GS3DC_OK;
}

int gs3dc_get_gradients(gs3dc_ctx* c, float* d_raw_positions, float* d_raw_scales, float* d_raw_rotations,
                        float* d_raw_sh_coeffs, float* d_raw_opacities) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (!c->have_step_grads)
        return fail(c, GS3DC_ERR_STATE, "no gradients kept: run gs3dc_train_step with GS3DC_OPT_KEEP_GRADIENTS");
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->N;
    int rc;
    if ((rc = download(c, d_raw_positions, c->g_pos.p, 3 * n * 4)) || (rc = download(c, d_raw_scales, c->g_sc.p, 3 * n * 4)) ||
        (rc = download(c, d_raw_rotations, c->g_rot.p, 4 * n * 4)) ||
        (rc = download(c, d_raw_sh_coeffs, c->g_sh.p, 3 * n * c->max_coeffs * 4)) ||
        (rc = download(c, d_raw_opacities, c->g_op.p, n * 4)))
        return rc;
    return gs3dc_synchronize(c);
}

int gs3dc_get_image(gs3dc_ctx* c, float* image) {
    if (!c || !image) return GS3DC_ERR_INVALID_ARG;
    if (c->W <= 0 || !c->image.p) return fail(c, GS3DC_ERR_STATE, "nothing has been rendered");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(image, c->image.p, (size_t)c->W * c->H * 3 * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_get_batch_image(gs3dc_ctx* c, int view, float* image) {
    if (!c || !image) return GS3DC_ERR_INVALID_ARG;
    auto& b = c->batch;
    if (b.view_pix.size() < 2 || !b.image.p) return fail(c, GS3DC_ERR_STATE, "no multi-view step has run");
    const int nv = (int)b.view_pix.size() - 1;
    if (view < 0 || view >= nv) return fail(c, GS3DC_ERR_INVALID_ARG, "view %d outside 0..%d", view, nv - 1);
    CK(cudaSetDevice(c->device));
    const unsigned long long p0 = b.view_pix[view], p1 = b.view_pix[view + 1];
    CK(cudaMemcpyAsync(image, b.image.p + 3 * p0, (size_t)(p1 - p0) * 3 * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_get_raw_params(gs3dc_ctx* c, gs3d_raw_params* r) {
    if (!c || !r) return GS3DC_ERR_INVALID_ARG;
    int rc = require_model(c);
    if (rc) return rc;
    if (!c->model_raw) return fail(c, GS3DC_ERR_STATE, "the device model is an activated render model");
    if (r->count != c->N || r->max_coeffs != c->max_coeffs)
        return fail(c, GS3DC_ERR_INVALID_ARG, "host params have N=%d mc=%d, device N=%d mc=%d", r->count,
                    r->max_coeffs, c->N, c->max_coeffs);
    const size_t n = (size_t)c->N;
    if (chosen_form(c) && (rc = unload_chosen(c))) return rc;
    if ((rc = download(c, r->raw_positions, c->pos.p, 3 * n * 4))) return rc;
    if ((rc = download(c, r->raw_scales, c->sc.p, 3 * n * 4))) return rc;
    if ((rc = download(c, r->raw_rotations, c->rot.p, 4 * n * 4))) return rc;
    if ((rc = download(c, r->raw_sh_coeffs, c->sh.p, 3 * n * c->max_coeffs * 4))) return rc;
    if ((rc = download(c, r->raw_opacities, c->op.p, n * 4))) return rc;
    return gs3dc_synchronize(c);
}

int gs3dc_preprocess(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg,
                     const gs3dc_screen_arrays* out) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_preprocess")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg, true)) || (rc = require_model(c))) return rc;
    CK(cudaSetDevice(c->device));
    const bool cache = !cfg->eval_3D && out &&
                       (out->cov3D || out->p_view || out->p_hom_w || out->cov2D || out->cov2D_det);
    if ((rc = run_preprocess(c, cam, cfg, cache))) return rc;
    if (out) {
        const size_t n = (size_t)c->N;
        CK(c->x_means2D.ensure(2 * n));
        CK(c->x_depths.ensure(n));
        CK(c->x_conics.ensure(3 * n));
        CK(c->x_opac.ensure(n));
        CK(c->x_rgb.ensure(3 * n));
        CK(c->x_radii.ensure(n));
        CK(c->x_tiles.ensure(n));
        ScreenArrays a{c->x_means2D.p, c->x_depths.p, c->x_conics.p, c->x_opac.p, c->x_rgb.p, c->x_radii.p, c->x_tiles.p};
        CK(launch_export_screen(c->stream, c->N, screen_ptrs(c, false), a));
        if ((rc = download(c, out->means2D, a.means2D, 2 * n * 4)) || (rc = download(c, out->depths, a.depths, n * 4)) ||
            (rc = download(c, out->conics, a.conics, 3 * n * 4)) ||
            (rc = download(c, out->opacities_2d, a.opac2d, n * 4)) || (rc = download(c, out->rgb, a.rgb, 3 * n * 4)) ||
            (rc = download(c, out->radii, a.radii, n * 4)) || (rc = download(c, out->tiles_touched, a.tiles, n * 4)))
            return rc;
        if (c->mode_e3 && ((rc = download(c, out->gauss2screen, c->e3_g2s.p, 16 * n * 4)) ||
                           (rc = download(c, out->cov3D_inv, c->e3_ci.p, 6 * n * 4)) ||
                           (rc = download(c, out->mean_offset, c->e3_mo.p, 3 * n * 4))))
            return rc;
        if (cache) {
            if ((rc = download(c, out->cov3D, c->c_cov3D.p, 6 * n * 4)) ||
                (rc = download(c, out->p_view, c->c_pview.p, 3 * n * 4)) ||
                (rc = download(c, out->p_hom_w, c->c_phw.p, n * 4)) ||
                (rc = download(c, out->cov2D, c->c_cov2D.p, 3 * n * 4)) ||
                (rc = download(c, out->cov2D_det, c->c_det.p, n * 4)))
                return rc;
        }
    }
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_bin(gs3dc_ctx* c, int num_gaussians, const gs3dc_screen_arrays* in, const gs3d_camera* cam,
              const gs3d_render_config* cfg, int64_t* total_pairs, uint64_t* keys_unsorted,
              uint32_t* values_unsorted) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_bin")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg, true))) return rc;
    CK(cudaSetDevice(c->device));
    if (!in) {
        if (!c->have_pairs) return fail(c, GS3DC_ERR_STATE, "gs3dc_bin without arrays needs gs3dc_preprocess first");
    } else {
        if (num_gaussians < 0) return fail(c, GS3DC_ERR_INVALID_ARG, "negative num_gaussians");
        if (num_gaussians > 0 && (!in->means2D || !in->depths || !in->radii || !in->tiles_touched))
            return fail(c, GS3DC_ERR_INVALID_ARG, "means2D, depths, radii and tiles_touched are required");
        if (num_gaussians > 0 && cfg->eval_3D && (!in->cov3D_inv || !in->mean_offset))
            return fail(c, GS3DC_ERR_INVALID_ARG, "eval_3D binning needs cov3D_inv and mean_offset");
        // the binned set replaces the device model's pairs; per-Gaussian records are not needed
        const size_t n = (size_t)num_gaussians;
        if ((rc = ensure_ctrl(c, num_gaussians))) return rc;
        CK(c->x_means2D.ensure(2 * n));
        CK(c->x_depths.ensure(n));
        CK(c->x_radii.ensure(n));
        CK(c->x_tiles.ensure(n));
        if ((rc = ensure_pixels(c, cam->width, cam->height))) return rc;
        if (n) {
            CK(cudaMemcpyAsync(c->x_means2D.p, in->means2D, 2 * n * 4, cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(c->x_depths.p, in->depths, n * 4, cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(c->x_radii.p, in->radii, n * 4, cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(c->x_tiles.p, in->tiles_touched, n * 4, cudaMemcpyHostToDevice, c->stream));
        }
        long long total = 0;
        for (size_t i = 0; i < n; i++) total += in->tiles_touched[i];
        if ((rc = ensure_pairs(c, (unsigned long long)total > c->cap ? (unsigned long long)total : c->cap, c->num_tiles)))
            return rc;
        if ((rc = push_params(c, cam, cfg, nullptr, 0, nullptr))) return rc;
        CK(cudaMemsetAsync(c->ctrl_region.p, 0, ctrl_bytes_for(num_gaussians), c->stream));
        if (total > 0) {
            // unwritten slots (malformed tiles_touched) read as zero keys
            CK(cudaMemsetAsync(c->keys[0].p, 0, (size_t)total * 8, c->stream));
            CK(cudaMemsetAsync(c->vals[0].p, 0, (size_t)total * 4, c->stream));
        }
        ScreenArrays a{c->x_means2D.p, c->x_depths.p, nullptr, nullptr, nullptr, c->x_radii.p, c->x_tiles.p};
        PairPtrs pr{c->keys[0].p, c->vals[0].p, c->cap, c->scan_desc};
        c->mode_e3 = cfg->eval_3D;
        if (c->mode_e3) {
            // per-tile depth keys from the caller's inverse covariances and mean offsets
            if ((rc = ensure_e3(c, num_gaussians))) return rc;
            if (n) {
                CK(cudaMemcpyAsync(c->e3_ci.p, in->cov3D_inv, 6 * n * 4, cudaMemcpyHostToDevice, c->stream));
                CK(cudaMemcpyAsync(c->e3_mo.p, in->mean_offset, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
            }
            CK(launch_e3_view(c->stream, c->sp_dev, c->num_tiles, e3_ptrs(c)));
            CK(launch_bin_arrays_e3(c->stream, c->sp_dev, num_gaussians, a, e3_ptrs(c), pr, c->ctrl));
        } else {
            CK(launch_bin_arrays(c->stream, c->sp_dev, num_gaussians, a, pr, c->ctrl));
        }
        if ((rc = read_control(c))) return rc;
        c->have_pairs = true;
        c->have_screen = false;  // the pairs no longer belong to the device model
        c->have_sorted = c->have_raster = c->have_rgrad = false;
    }
    if (total_pairs) *total_pairs = (int64_t)c->last_pairs;
    const size_t P = (size_t)c->last_pairs;
    if ((rc = download(c, keys_unsorted, c->keys[0].p, P * 8))) return rc;
    if ((rc = download(c, values_unsorted, c->vals[0].p, P * 4))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_sort(gs3dc_ctx* c, uint64_t* keys_sorted, uint32_t* values_sorted, uint32_t* tile_ranges) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (!c->have_pairs) return fail(c, GS3DC_ERR_STATE, "gs3dc_sort needs pairs (gs3dc_preprocess or gs3dc_bin)");
    CK(cudaSetDevice(c->device));
    c->kernels_last = 0;
    const bool timing = c->stage_timing;
    c->stage_timing = false;
    int rc = seq_sort_scratch(c);
    if (!rc) rc = seq_sort(c);
    c->stage_timing = timing;
    if (rc) return rc;
    if ((rc = read_control(c))) return rc;
    const size_t P = (size_t)c->last_pairs;
    const int w = c->sorted_which;
    if ((rc = download(c, keys_sorted, c->keys[w].p, P * 8)) || (rc = download(c, values_sorted, c->vals[w].p, P * 4)) ||
        (rc = download(c, tile_ranges, c->ranges.p, 2 * (size_t)c->num_tiles * 4)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_sorted = true;
    return GS3DC_OK;
}

int gs3dc_sort_pairs(gs3dc_ctx* c, int64_t total_pairs, const uint64_t* keys, const uint32_t* values, int num_tiles,
                     uint64_t* keys_sorted, uint32_t* values_sorted, uint32_t* tile_ranges) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (total_pairs < 0 || num_tiles <= 0 || (total_pairs > 0 && (!keys || !values)))
        return fail(c, GS3DC_ERR_INVALID_ARG, "bad pair input (P=%lld, tiles=%d)", (long long)total_pairs, num_tiles);
    CK(cudaSetDevice(c->device));
    const size_t P = (size_t)total_pairs;
    for (size_t i = 0; i < P; i++)
        if ((keys[i] >> 32) >= (uint64_t)num_tiles)
            return fail(c, GS3DC_ERR_INVALID_ARG, "key %zu has tile %llu >= num_tiles %d", i,
                        (unsigned long long)(keys[i] >> 32), num_tiles);
    int rc;
    CK(c->ranges.ensure(2 * (size_t)num_tiles));
    CK(c->tile_order.ensure((size_t)num_tiles));
    c->num_tiles = num_tiles;
    if ((rc = ensure_pairs(c, P > c->cap ? P : c->cap, num_tiles))) return rc;
    // the sort reads only spin_limit from the parameters
    const int slot = c->sp_slot;
    c->sp_slot = (c->sp_slot + 1) % kParamSlots;
    CK(cudaEventSynchronize(c->sp_event[slot]));
    std::memset(&c->sp_ring[slot], 0, sizeof(StepParams));
    c->sp_ring[slot].spin_limit = c->spin_limit;
    CK(cudaMemcpyAsync(c->sp_dev, &c->sp_ring[slot], sizeof(StepParams), cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->sp_event[slot], c->stream));
    CK(cudaMemsetAsync(c->ctrl_region.p, 0, sizeof(Control), c->stream));
    unsigned long long P64 = (unsigned long long)P;
    CK(cudaMemcpyAsync(&c->ctrl->total_pairs, &P64, 8, cudaMemcpyHostToDevice, c->stream));
    if (P) {
        CK(cudaMemcpyAsync(c->keys[0].p, keys, P * 8, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->vals[0].p, values, P * 4, cudaMemcpyHostToDevice, c->stream));
    }
    c->have_pairs = true;
    c->have_screen = false;
    CK(cudaStreamSynchronize(c->stream));
    return gs3dc_sort(c, keys_sorted, values_sorted, tile_ranges);
}

int gs3dc_rasterize(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg, float* image,
                    float* T_final, int* n_contrib) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_rasterize")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg, true))) return rc;
    if (!c->have_sorted || !c->have_screen)
        return fail(c, GS3DC_ERR_STATE, "gs3dc_rasterize needs gs3dc_preprocess and gs3dc_sort of the model");
    if (cfg->eval_3D != c->mode_e3)
        return fail(c, GS3DC_ERR_STATE, "eval_3D differs between gs3dc_preprocess and gs3dc_rasterize");
    if (cam->width != c->W || cam->height != c->H)
        return fail(c, GS3DC_ERR_INVALID_ARG, "camera size differs from the preprocessed one");
    CK(cudaSetDevice(c->device));
    if ((rc = push_params(c, cam, cfg, nullptr, 0, nullptr))) return rc;
    const int w = c->sorted_which;
    if (c->mode_e3)
        CK(launch_raster_e3(c->stream, c->sp_dev, c->num_tiles, c->ranges.p, c->tile_order.p, c->vals[w].p,
                            e3_ptrs(c), pixel_ptrs(c), c->ctrl));
    else
        CK(launch_raster_fwd_plain(c->stream, c->sp_dev, c->num_tiles, false, c->ranges.p, c->tile_order.p,
                                   c->vals[w].p, screen_ptrs(c, false), pixel_ptrs(c), c->ctrl));
    const size_t np = (size_t)c->W * c->H;
    if ((rc = download(c, image, c->image.p, 3 * np * 4)) || (rc = download(c, T_final, c->T_final.p, np * 4)) ||
        (rc = download(c, n_contrib, c->n_contrib.p, np * 4)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_raster = true;
    return GS3DC_OK;
}

int gs3dc_rasterize_arrays(gs3dc_ctx* c, int num_gaussians, const gs3dc_screen_arrays* in, int64_t total_pairs,
                           const uint32_t* values_sorted, int num_tiles, const uint32_t* tile_ranges,
                           const gs3d_camera* cam, const gs3d_render_config* cfg, float* image, float* T_final,
                           int* n_contrib) {
    if (!c || !in || !tile_ranges) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_rasterize_arrays")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg))) return rc;   // the 3D mode needs its own per-Gaussian arrays
    const int gx = (cam->width + kTile - 1) / kTile, gy = (cam->height + kTile - 1) / kTile;
    if (num_gaussians < 0 || total_pairs < 0 || num_tiles != gx * gy)
        return fail(c, GS3DC_ERR_INVALID_ARG, "bad sizes: N=%d, P=%lld, %d tiles (the camera has %d)", num_gaussians,
                    (long long)total_pairs, num_tiles, gx * gy);
    if (num_gaussians > 0 && (!in->means2D || !in->conics || !in->opacities_2d || !in->rgb))
        return fail(c, GS3DC_ERR_INVALID_ARG, "means2D, conics, opacities_2d and rgb are required");
    if (total_pairs > 0 && !values_sorted) return fail(c, GS3DC_ERR_INVALID_ARG, "values_sorted is required");
    if ((unsigned long long)total_pairs > 0xFFFFFFFFull)
        return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "%lld pairs exceed the 32-bit tile-range format", (long long)total_pairs);
    // every index the rasteriser will follow must stay inside the caller's arrays
    const size_t P = (size_t)total_pairs, n = (size_t)num_gaussians;
    for (size_t j = 0; j < P; j++)
        if (values_sorted[j] >= n)
            return fail(c, GS3DC_ERR_INVALID_ARG, "values_sorted[%zu] = %u is not below N = %d", j, values_sorted[j],
                        num_gaussians);
    for (int t = 0; t < num_tiles; t++)
        if (tile_ranges[2 * t] > tile_ranges[2 * t + 1] || tile_ranges[2 * t + 1] > P)
            return fail(c, GS3DC_ERR_INVALID_ARG, "tile %d has range [%u, %u) outside [0, %zu)", t, tile_ranges[2 * t],
                        tile_ranges[2 * t + 1], P);
    CK(cudaSetDevice(c->device));
    if ((rc = ensure_pixels(c, cam->width, cam->height))) return rc;
    const size_t nn = n ? n : 1;
    if (nn > c->rec0.n || nn > c->rec1.n || nn > c->cbt.n) drop_graphs(c);
    CK(c->rec0.ensure(nn));
    CK(c->rec1.ensure(nn));
    CK(c->cbt.ensure(nn));
    CK(c->dm2.ensure(2 * nn));
    CK(c->dcon.ensure(3 * nn));
    CK(c->drgb.ensure(3 * nn));
    CK(c->dop.ensure(nn));
    CK(c->x_means2D.ensure(2 * nn));
    CK(c->x_conics.ensure(3 * nn));
    CK(c->x_opac.ensure(nn));
    CK(c->x_rgb.ensure(3 * nn));
    if (n) {
        CK(cudaMemcpyAsync(c->x_means2D.p, in->means2D, 2 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->x_conics.p, in->conics, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->x_opac.p, in->opacities_2d, n * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->x_rgb.p, in->rgb, 3 * n * 4, cudaMemcpyHostToDevice, c->stream));
    }
    ScreenArrays a{c->x_means2D.p, nullptr, c->x_conics.p, c->x_opac.p, c->x_rgb.p, nullptr, nullptr};
    CK(launch_import_screen(c->stream, num_gaussians, a, screen_ptrs(c, false)));
    if ((rc = ensure_pairs(c, P > c->cap ? P : c->cap, c->num_tiles))) return rc;
    if (P) CK(cudaMemcpyAsync(c->vals[0].p, values_sorted, P * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->ranges.p, tile_ranges, 2 * (size_t)num_tiles * 4, cudaMemcpyHostToDevice, c->stream));
    CK(launch_tile_order(c->stream, c->ranges.p, c->num_tiles, c->tile_order.p));
    c->sorted_which = 0;
    c->screen_n = num_gaussians;
    c->screen_imported = true;
    c->mode_e3 = false;
    c->have_screen = c->have_sorted = true;
    c->have_pairs = c->have_raster = c->have_rgrad = false;
    if ((rc = push_params(c, cam, cfg, nullptr, 0, nullptr))) return rc;
    CK(launch_raster_fwd_plain(c->stream, c->sp_dev, c->num_tiles, false, c->ranges.p, c->tile_order.p, c->vals[0].p,
                               screen_ptrs(c, false), pixel_ptrs(c), c->ctrl));
    const size_t np = (size_t)c->W * c->H;
    if ((rc = download(c, image, c->image.p, 3 * np * 4)) || (rc = download(c, T_final, c->T_final.p, np * 4)) ||
        (rc = download(c, n_contrib, c->n_contrib.p, np * 4)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_raster = true;
    return GS3DC_OK;
}

int gs3dc_render(gs3dc_ctx* c, const gs3d_gaussians* g, const gs3d_camera* cam, const gs3d_render_config* cfg,
                 float* image) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_render")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg, true))) return rc;
    if (g && (rc = gs3dc_set_gaussians(c, g))) return rc;
    if ((rc = require_model(c))) return rc;
    if ((rc = gs3dc_preprocess(c, cam, cfg, nullptr))) return rc;
    long long k0 = c->kernels_last;
    if ((rc = gs3dc_sort(c, nullptr, nullptr, nullptr))) return rc;
    k0 += c->kernels_last;
    if ((rc = gs3dc_rasterize(c, cam, cfg, image, nullptr, nullptr))) return rc;
    c->kernels_last = k0 + 1;
    return GS3DC_OK;
}

int gs3dc_raster_backward(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg, const float* d_image,
                          float* d_means2D, float* d_conics, float* d_rgb, float* d_opacities_2d) {
    if (!c || !d_image) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_raster_backward")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg))) return rc;
    if (!c->have_raster) return fail(c, GS3DC_ERR_STATE, "gs3dc_raster_backward needs gs3dc_rasterize first");
    CK(cudaSetDevice(c->device));
    const size_t np = (size_t)c->W * c->H, n = (size_t)c->screen_n;
    CK(c->d_image.ensure(3 * np));
    CK(cudaMemcpyAsync(c->d_image.p, d_image, 3 * np * 4, cudaMemcpyHostToDevice, c->stream));
    if ((rc = push_params(c, cam, cfg, nullptr, 0, nullptr))) return rc;
    CK(cudaMemsetAsync(c->dm2.p, 0, 2 * n * 4, c->stream));
    CK(cudaMemsetAsync(c->dcon.p, 0, 3 * n * 4, c->stream));
    CK(cudaMemsetAsync(c->drgb.p, 0, 3 * n * 4, c->stream));
    CK(cudaMemsetAsync(c->dop.p, 0, n * 4, c->stream));
    const int w = c->sorted_which;
    CK(launch_raster_bwd_plain(c->stream, c->sp_dev, c->num_tiles, false, c->ranges.p, c->tile_order.p, c->vals[w].p,
                               screen_ptrs(c, false), pixel_ptrs(c), rgrad_ptrs(c), c->ctrl));
    if ((rc = download(c, d_means2D, c->dm2.p, 2 * n * 4)) || (rc = download(c, d_conics, c->dcon.p, 3 * n * 4)) ||
        (rc = download(c, d_rgb, c->drgb.p, 3 * n * 4)) || (rc = download(c, d_opacities_2d, c->dop.p, n * 4)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_rgrad = true;
    return GS3DC_OK;
}

int gs3dc_preprocess_backward(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg,
                              const float* raw_rotations, float* d_raw_positions, float* d_raw_scales,
                              float* d_raw_rotations, float* d_raw_sh_coeffs, float* d_raw_opacities) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_preprocess_backward")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg))) return rc;
    if (c->screen_imported)
        return fail(c, GS3DC_ERR_STATE, "gs3dc_preprocess_backward needs the device model's own forward "
                                        "(the screen records came from gs3dc_rasterize_arrays)");
    if (!c->have_rgrad) return fail(c, GS3DC_ERR_STATE, "gs3dc_preprocess_backward needs gs3dc_raster_backward");
    if (!c->model_raw && !raw_rotations)
        return fail(c, GS3DC_ERR_INVALID_ARG, "an activated device model needs the raw rotations");
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->N;
    if ((rc = ensure_grads(c))) return rc;
    const float* raw_rot_dev = nullptr;
    if (!c->model_raw) {
        CK(c->raw_rot_tmp.ensure(4 * n));
        CK(cudaMemcpyAsync(c->raw_rot_tmp.p, raw_rotations, 4 * n * 4, cudaMemcpyHostToDevice, c->stream));
        raw_rot_dev = c->raw_rot_tmp.p;
    }
    const size_t mc3 = (size_t)c->max_coeffs * 3;
    if ((rc = push_params(c, cam, cfg, nullptr, 0, nullptr, raw_rot_dev))) return rc;
    CK(launch_preprocess_bwd_plain(c->stream, c->sp_dev, c->N, c->max_coeffs * 3, 0, model_ptrs(c), adam_ptrs(c),
                                   screen_ptrs(c, false), rgrad_ptrs(c), grad_ptrs(c), c->ctrl));
    if ((rc = download(c, d_raw_positions, c->g_pos.p, 3 * n * 4)) ||
        (rc = download(c, d_raw_scales, c->g_sc.p, 3 * n * 4)) ||
        (rc = download(c, d_raw_rotations, c->g_rot.p, 4 * n * 4)) ||
        (rc = download(c, d_raw_sh_coeffs, c->g_sh.p, mc3 * n * 4)) ||
        (rc = download(c, d_raw_opacities, c->g_op.p, n * 4)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_grads = true;
    return GS3DC_OK;
}

int gs3dc_optimizer_step(gs3dc_ctx* c, const gs3d_train_config* tc, int iteration) {
    if (!c || !tc) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_optimizer_step")) return rc_;
    if (!c->have_grads) return fail(c, GS3DC_ERR_STATE, "gs3dc_optimizer_step needs gs3dc_preprocess_backward");
    CK(cudaSetDevice(c->device));
    int rc;
    if ((rc = ensure_adam(c))) return rc;
    if (tc->use_adam) c->adam_step++;
    gs3d_camera cam{};
    cam.width = c->W > 0 ? c->W : 1;
    cam.height = c->H > 0 ? c->H : 1;
    cam.tan_fovx = cam.tan_fovy = 1.0f;
    gs3d_render_config cfg{};
    cfg.tile_w = cfg.tile_h = kTile;
    cfg.scale_modifier = 1.0f;
    if ((rc = push_params(c, &cam, &cfg, tc, iteration, nullptr))) return rc;
    CK(launch_optimizer_plain(c->stream, c->sp_dev, c->N, c->max_coeffs * 3, model_ptrs(c), adam_ptrs(c), grad_ptrs(c),
                              nullptr));
    CK(cudaStreamSynchronize(c->stream));
    c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
    return GS3DC_OK;
}

int gs3dc_selftest_bounded_wait(gs3dc_ctx* c, uint32_t spin_limit) {
    if (!c || spin_limit == 0 || spin_limit > (1u << 24)) return GS3DC_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    // two zeroed descriptors at the head of the scan-descriptor area, status word cleared
    CK(cudaMemsetAsync(c->ctrl_region.p, 0, ctrl_bytes_for(2 * kBlock), c->stream));
    CK(launch_wait_selftest(c->stream, c->scan_desc, &c->ctrl->status, spin_limit));
    const int rc = read_control(c);
    CK(cudaMemsetAsync(c->ctrl_region.p, 0, ctrl_bytes_for(2 * kBlock), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return rc;
}

int gs3dc_get_stage_times(gs3dc_ctx* c, float* ms, int n_stages) {
    if (!c || !ms || n_stages < 0) return GS3DC_ERR_INVALID_ARG;
    for (int k = 0; k < n_stages && k < GS3DC_NUM_STAGES; k++) ms[k] = c->stage_ms[k];
    return GS3DC_OK;
}

// Acknowledges a sticky overflow: the Adam step counter follows the updates
// the device actually applied, and later steps may update again.
int acknowledge_overflow(gs3dc_ctx* c) {
    c->adam_step = (int)c->persist_host->applied_steps;
    c->persist_host->sticky_overflow = 0;
    CK(cudaMemsetAsync(&c->persist->sticky_overflow, 0, sizeof(unsigned), c->stream));
    return GS3DC_OK;
}

int gs3dc_synchronize(gs3dc_ctx* c) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    int rc = read_control(c);
    if (rc) return rc;
    c->pending_check = false;
    if (c->persist_host->sticky_overflow) {
        if ((rc = acknowledge_overflow(c))) return rc;
        return fail(c, GS3DC_ERR_PAIR_OVERFLOW,
                    "a train step found more tile pairs than the capacity of %llu; it and the steps queued "
                    "after it were skipped (%llu optimiser steps applied)",
                    c->cap, (unsigned long long)c->persist_host->applied_steps);
    }
    return GS3DC_OK;
}

int gs3dc_train_step(gs3dc_ctx* c, const gs3d_camera* cam, const float* gt, int gt_on_device,
                     const gs3d_render_config* cfg, const gs3d_train_config* tc, int iteration, float* loss) {
    if (!c || !gt || !tc) return GS3DC_ERR_INVALID_ARG;
    int rc;
    if ((rc = check_config(c, cam, cfg)) || (rc = require_model(c))) return rc;
    if (!c->model_raw) return fail(c, GS3DC_ERR_STATE, "gs3dc_train_step needs a raw model (gs3dc_set_raw_params)");
    CK(cudaSetDevice(c->device));
    if ((rc = ensure_adam(c))) return rc;
    if ((rc = ensure_grads(c))) return rc;
    if ((rc = ensure_depth_sort(c))) return rc;
    if (chosen_form(c) && !c->chosen_ready) return fail(c, GS3DC_ERR_NO_MODEL, "no reduced-storage model loaded");
    if ((rc = ensure_pixels(c, cam->width, cam->height))) return rc;
    const size_t np = (size_t)cam->width * cam->height;
    const float* gt_dev = gt;
    const bool host_gt = !gt_on_device;
    int gslot = 0;
    if (host_gt) {
        // the copy runs on its own stream, overlapping the front half of the step; buffer gslot
        // is reused only after the step that last read it has passed its back half
        gslot = c->gt_slot;
        c->gt_slot ^= 1;
        CK(c->gtb[gslot].ensure(3 * np));
        if (c->gt_free_recorded[gslot]) CK(cudaStreamWaitEvent(c->copy_stream, c->ev_gt_free[gslot], 0));
        CK(cudaMemcpyAsync(c->gtb[gslot].p, gt, 3 * np * 4, cudaMemcpyHostToDevice, c->copy_stream));
        CK(cudaEventRecord(c->ev_gt_ready, c->copy_stream));
        gt_dev = c->gtb[gslot].p;
    }
    // a shape's first step runs synchronously (an overflow of the pair-capacity guess is redone at
    // once); later steps of a shape replay its graphs
    const long long shape[6] = {c->N, c->max_coeffs, cam->width, cam->height, c->form, c->sort_mode};
    bool first = c->cap == 0 || !shape_seen(c, shape);
    if (c->cap == 0 || c->sort_num_tiles != c->num_tiles) {
        unsigned long long guess = c->min_cap ? c->min_cap : (unsigned long long)c->N * 8ull;
        if ((rc = ensure_pairs(c, guess > c->cap ? guess : c->cap, c->num_tiles))) return rc;
    }
    const int step_before = c->adam_step;
    const long long tkey[6] = {c->N, cam->width, cam->height, c->form, c->sort_mode, c->fused_adam ? 1 : 0};
    const bool tuning = tune_begin(c, tune_slot(c, tkey), tkey);
    const bool user_timing = c->stage_timing;
    if (tuning) c->stage_timing = true;   // the trial step runs un-captured with events between stages
    struct RestoreTiming {
        gs3dc_ctx* c;
        bool v;
        ~RestoreTiming() { c->stage_timing = v; }
    } restore_timing{c, user_timing};
    // a target from host memory: the forward runs before its copy has landed (front half) and the
    // L1 follows in the back half, so the copy overlaps the forward too; timed steps keep the fused
    // L1 (the stage events would count the wait)
    const bool loss_later = host_gt && !c->stage_timing;
    for (int attempt = 0; attempt < 3; attempt++) {
        c->adam_step = step_before + (tc->use_adam ? 1 : 0);
        if ((rc = push_params(c, cam, cfg, tc, iteration, gt_dev))) return rc;
        const long long key[kGraphKey] = {
            c->N, c->max_coeffs, cam->width, cam->height, (long long)c->cap, c->sort_passes,
            (long long)c->spin_limit,
            (c->fused_adam ? 1 : 2) + 4 * c->sort_mode + 16 * c->form + 64 * (c->keep_grads ? 1 : 0) +
                128 * c->fwd_ppt + 1024 * c->bwd_ppt + 8192 * c->fwd_batch + 8192 * 512 * c->bwd_batch +
                (loss_later ? 1ll << 40 : 0ll),
            (long long)g_alloc_epoch.load(std::memory_order_relaxed)};
        c->kernels_last = 0;
        if (c->use_graph && !c->stage_timing && !first && attempt == 0) {
            gs3dc_ctx::GraphSlot* slot = find_slot(c, key);
            if (!slot) {
                slot = victim_slot(c);
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                rc = seq_train_front(c, loss_later);
                cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
                if (rc) return rc;
                CK(ec);
                cudaError_t ei = cudaGraphInstantiate(&slot->front, g, 0);
                cudaGraphDestroy(g);
                CK(ei);
                CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                rc = seq_train_back(c, loss_later);
                ec = cudaStreamEndCapture(c->stream, &g);
                if (rc) {
                    drop_slot(*slot);
                    return rc;
                }
                if (ec != cudaSuccess) drop_slot(*slot);
                CK(ec);
                ei = cudaGraphInstantiate(&slot->back, g, 0);
                cudaGraphDestroy(g);
                if (ei != cudaSuccess) drop_slot(*slot);
                CK(ei);
                std::memcpy(slot->key, key, sizeof(key));
                slot->kernels = c->kernels_last;
                c->graph_captures++;
            }
            slot->used = ++c->gclock;
            c->kernels_last = slot->kernels;
            CK(cudaGraphLaunch(slot->front, c->stream));
            if (host_gt) CK(cudaStreamWaitEvent(c->stream, c->ev_gt_ready, 0));
            CK(cudaGraphLaunch(slot->back, c->stream));
            c->graph_replays++;
        } else {
            if ((rc = seq_train_front(c, loss_later))) return rc;
            if (host_gt) CK(cudaStreamWaitEvent(c->stream, c->ev_gt_ready, 0));
            if ((rc = seq_train_back(c, loss_later))) return rc;
        }
        if (host_gt) {
            CK(cudaEventRecord(c->ev_gt_free[gslot], c->stream));
            c->gt_free_recorded[gslot] = true;
        }
        c->have_step_grads = c->keep_grads;
        if (!loss && !first && !c->stage_timing) {
            c->pending_check = true;  // overflow is reported by the next synchronising call
            return GS3DC_OK;
        }
        if ((rc = read_control(c))) {
            c->adam_step = step_before;
            return rc;
        }
        if (c->persist_host->sticky_overflow) {
            // nothing was updated: the backward and the optimiser skip overflowed steps
            if ((rc = acknowledge_overflow(c))) return rc;
            const unsigned long long P = c->ctrl_host->total_pairs;
            if (!(c->ctrl_host->status & kStatusOverflow)) {
                // an earlier asynchronous step overflowed: report it, this step was skipped too
                return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "an earlier queued train step overflowed the pair capacity");
            }
            if ((rc = ensure_pairs(c, P + P / 2 + 4096, c->num_tiles))) return rc;
            first = true;
            continue;
        }
        mark_shape_seen(c, shape);   // the capacity holds this shape's pairs
        if (loss) *loss = (float)(c->ctrl_host->loss_sum / (double)(3.0 * (double)np));
        if (c->stage_timing) {
            for (int k = 0; k < GS3DC_NUM_STAGES; k++)
                CK(cudaEventElapsedTime(&c->stage_ms[k], c->stage_ev[k], c->stage_ev[k + 1]));
        }
        if (tuning)
            tune_end(c, tune_slot(c, tkey), c->stage_ms[GS3DC_STAGE_RASTER_FWD], c->stage_ms[GS3DC_STAGE_RASTER_BWD]);
        return GS3DC_OK;
    }
    c->adam_step = step_before;
    return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "tile-pair capacity kept overflowing");
}

int gs3dc_train_step_batch(gs3dc_ctx* c, int n_views, const gs3d_camera* cams, const float* gt, int gt_on_device,
                           const gs3d_render_config* cfg, const gs3d_train_config* tc, int iteration, float* loss) {
    if (!c || !cams || !gt || !cfg || !tc) return GS3DC_ERR_INVALID_ARG;
    if (n_views < 1 || n_views > kMaxBatchViews)
        return fail(c, GS3DC_ERR_INVALID_ARG, "n_views %d outside 1..%d", n_views, kMaxBatchViews);
    int rc;
    if ((rc = require_model(c))) return rc;
    if (!chosen_form(c) || !c->chosen_ready)
        return fail(c, GS3DC_ERR_STATE, "multi-view steps run in the reduced-storage form (GS3DC_FORM_BF16 / _FP16)");
    for (int v = 0; v < n_views; v++)
        if ((rc = check_config(c, &cams[v], cfg))) return rc;
    CK(cudaSetDevice(c->device));
    auto& b = c->batch;
    BatchShape sh;
    sh.V = n_views;
    sh.VN = (long long)c->N * n_views;
    sh.seg = ((long long)c->N + 8191) / 8192 * 8192;
    sh.VS = sh.seg * n_views;
    if (sh.VS >= (1LL << 31)) return fail(c, GS3DC_ERR_INVALID_ARG, "%lld (view, Gaussian) entries exceed 2^31", sh.VN);
    std::vector<unsigned> tile_base(n_views), pix_base(n_views);
    unsigned long long tiles = 0, pix = 0, max_view_tiles = 0;
    b.view_pix.clear();
    for (int v = 0; v < n_views; v++) {
        const int gx = (cams[v].width + cfg->tile_w - 1) / cfg->tile_w, gy = (cams[v].height + cfg->tile_h - 1) / cfg->tile_h;
        tile_base[v] = (unsigned)tiles;
        pix_base[v] = (unsigned)pix;
        b.view_pix.push_back(pix);
        tiles += (unsigned long long)gx * gy;
        max_view_tiles = std::max(max_view_tiles, (unsigned long long)gx * gy);
        pix += (unsigned long long)cams[v].width * cams[v].height;
    }
    b.view_pix.push_back(pix);
    if (tiles >= (1ull << 24) || pix >= (1ull << 31))
        return fail(c, GS3DC_ERR_INVALID_ARG, "the views' %llu tiles / %llu pixels exceed 2^24 / 2^31", tiles, pix);
    sh.tiles = (unsigned)tiles;
    sh.pix = pix;
    // the pairs are sorted on the views' local tile ids
    sh.tile_digits = (bit_length(max_view_tiles > 1 ? (unsigned)(max_view_tiles - 1) : 0u) + 7) / 8;
    if ((rc = batch_buffers(c, sh))) return rc;
    if (c->keep_grads && (rc = ensure_grads(c))) return rc;
    const bool shape_new = b.cap == 0 || b.key[0] != c->N || b.key[1] != n_views || b.key[2] != (long long)sh.tiles ||
                           b.key[3] != (long long)sh.pix;
    if ((rc = batch_pairs(c, b.cap ? b.cap : (unsigned long long)sh.VN * 8ull + 4096ull, sh.tile_digits))) return rc;
    const float* gt_dev = gt;
    if (!gt_on_device) {
        CK(b.gt.ensure(3 * pix));
        CK(cudaMemcpyAsync(b.gt.p, gt, 3 * pix * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        gt_dev = b.gt.p;
    }
    if (!b.views_host) {
        CK(cudaMallocHost(&b.views_host, kMaxBatchViews * sizeof(StepParams)));
        CK(cudaEventCreateWithFlags(&b.views_event, cudaEventDisableTiming));
    }
    bool first = shape_new;
    const int step_before = c->adam_step;
    const long long tkey[6] = {c->N, n_views, (long long)sh.tiles, (long long)sh.pix, c->form, 1};
    const bool tuning = tune_begin(c, c->tune_batch, tkey);
    for (int attempt = 0; attempt < 3; attempt++) {
        c->adam_step = step_before + (tc->use_adam ? 1 : 0);
        CK(cudaEventSynchronize(b.views_event));   // the staging's previous copy has been consumed
        for (int v = 0; v < n_views; v++) {
            StepParams& p = b.views_host[v];
            fill_params(c, p, &cams[v], cfg, tc, iteration, gt_dev, nullptr);
            // each view's L1 mean enters the loss with weight 1 / n_views
            p.inv_n = 1.0f / ((float)n_views * 3.0f * (float)cams[v].width * (float)cams[v].height);
            p.tile_base = tile_base[v];
            p.pix_base = pix_base[v];
            p.sort_passes = kDepthDigits + sh.tile_digits;
        }
        CK(cudaMemcpyAsync(b.views.p, b.views_host, (size_t)n_views * sizeof(StepParams), cudaMemcpyHostToDevice,
                           c->stream));
        CK(cudaEventRecord(b.views_event, c->stream));
        const long long key[kGraphKey] = {
            c->N, n_views, (long long)sh.tiles, (long long)sh.pix, (long long)b.cap, c->form, (long long)c->spin_limit,
            c->max_coeffs + 1000 * (c->keep_grads ? 1 : 0) + 2000 * c->fwd_ppt + 20000 * c->bwd_ppt +
                200000LL * c->fwd_batch + 200000LL * 512 * c->bwd_batch,
            (long long)g_alloc_epoch.load(std::memory_order_relaxed)};
        if (c->use_graph && !first && !tuning && attempt == 0) {
            if (!b.graph || std::memcmp(key, b.key, sizeof(key)) != 0) {
                if (b.graph) cudaGraphExecDestroy(b.graph);
                b.graph = nullptr;
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                rc = seq_batch(c, sh);
                cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
                if (rc) return rc;
                CK(ec);
                CK(cudaGraphInstantiate(&b.graph, g, 0));
                cudaGraphDestroy(g);
                c->graph_captures++;
            }
            CK(cudaGraphLaunch(b.graph, c->stream));
            c->graph_replays++;
        } else {
            if ((rc = seq_batch(c, sh))) return rc;
        }
        std::memcpy(b.key, key, sizeof(key));
        c->have_step_grads = c->keep_grads;
        if (!loss && !first && !tuning) {
            c->pending_check = true;   // overflow is reported by the next synchronising call
            return GS3DC_OK;
        }
        if ((rc = read_control(c))) {
            c->adam_step = step_before;
            return rc;
        }
        if (c->persist_host->sticky_overflow) {
            if ((rc = acknowledge_overflow(c))) return rc;
            const unsigned long long P = c->ctrl_host->total_pairs;
            if (!(c->ctrl_host->status & kStatusOverflow))
                return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "an earlier queued train step overflowed the pair capacity");
            if ((rc = batch_pairs(c, P + P / 4 + 4096, sh.tile_digits))) return rc;
            first = true;
            continue;
        }
        if (loss) *loss = (float)c->ctrl_host->loss_sum;
        c->last_pairs = c->ctrl_host->total_pairs;
        if (tuning) {
            float f = 0.f, bw = 0.f;
            CK(cudaEventElapsedTime(&f, c->tune_ev[0], c->tune_ev[1]));
            CK(cudaEventElapsedTime(&bw, c->tune_ev[1], c->tune_ev[2]));
            tune_end(c, c->tune_batch, f, bw);
        }
        c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
        return GS3DC_OK;
    }
    c->adam_step = step_before;
    return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "tile-pair capacity kept overflowing");
}

int gs3dc_save_state(gs3dc_ctx* c, const char* path) {
    if (!c || !path) return GS3DC_ERR_INVALID_ARG;
    int rc;
    if ((rc = require_model(c))) return rc;
    if (!c->model_raw) return fail(c, GS3DC_ERR_STATE, "the device model is an activated render model");
    if (chosen_form(c) && !c->chosen_ready) return fail(c, GS3DC_ERR_STATE, "no reduced-storage model loaded");
    CK(cudaSetDevice(c->device));
    if ((rc = gs3dc_synchronize(c))) return rc;   // queued steps and their overflow bookkeeping first
    if ((rc = ensure_adam(c))) return rc;
    CkptHeader h{};
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = kCkptVersion;
    h.form = c->form;
    h.count = c->N;
    h.sh_degree = c->sh_degree;
    h.max_coeffs = c->max_coeffs;
    h.adam_step = c->adam_step;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(c, GS3DC_ERR_INVALID_ARG, "cannot open %s for writing", path);
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    std::vector<unsigned char> buf;
    const std::vector<void*> arrays = state_arrays(c);
    const std::vector<size_t> sizes = state_sizes(c->form, (size_t)c->N, (size_t)c->max_coeffs * 3);
    for (size_t k = 0; k < arrays.size() && ok; k++) {
        void* p = arrays[k];
        const size_t bytes = sizes[k];
        buf.resize(bytes);
        if (bytes && cudaMemcpy(buf.data(), p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(f);
            return fail(c, GS3DC_ERR_CUDA, "download of the training state failed");
        }
        ok = bytes == 0 || std::fwrite(buf.data(), 1, bytes, f) == bytes;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(c, GS3DC_ERR_INVALID_ARG, "write to %s failed", path);
    return GS3DC_OK;
}

int gs3dc_load_state(gs3dc_ctx* c, const char* path) {
    if (!c || !path) return GS3DC_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(c, GS3DC_ERR_INVALID_ARG, "cannot open %s", path);
    CkptHeader h{};
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0 ||
        h.version != kCkptVersion || h.count < 0 || h.max_coeffs < 1 || h.max_coeffs > 16 ||
        (h.form != GS3DC_FORM_PLAIN_FP32 && h.form != GS3DC_FORM_BF16 && h.form != GS3DC_FORM_FP16)) {
        std::fclose(f);
        return fail(c, GS3DC_ERR_INVALID_ARG, "%s is not a gs3dc training-state file", path);
    }
    // the file holds exactly the arrays its header describes: checked before the model is touched
    const size_t n = (size_t)h.count, mc3 = (size_t)h.max_coeffs * 3;
    const std::vector<size_t> sizes = state_sizes(h.form, n, mc3);
    size_t expect = sizeof(CkptHeader);
    for (size_t b : sizes) expect += b;
    if (std::fseek(f, 0, SEEK_END) != 0 || std::ftell(f) != (long)expect ||
        std::fseek(f, (long)sizeof(CkptHeader), SEEK_SET) != 0) {
        std::fclose(f);
        return fail(c, GS3DC_ERR_INVALID_ARG, "%s does not hold the %zu bytes its header describes", path, expect);
    }
    // the model's shape and form first (zeros), then every array from the file
    std::vector<float> z(std::max<size_t>(1, std::max(mc3, (size_t)4) * n), 0.0f);
    int rc = upload_model_arrays(c, h.count, h.sh_degree, h.max_coeffs, z.data(), z.data(), z.data(), z.data(),
                                 z.data());
    if (rc) {
        std::fclose(f);
        return rc;
    }
    c->model_raw = true;
    drop_graphs(c);
    c->form = h.form;
    c->chosen_ready = false;
    if ((rc = ensure_adam(c)) || (rc = zero_adam(c)) || (chosen_form(c) && (rc = load_chosen(c)))) {
        std::fclose(f);
        return rc;
    }
    CK(cudaStreamSynchronize(c->stream));
    std::vector<unsigned char> buf;
    const std::vector<void*> arrays = state_arrays(c);
    for (size_t k = 0; k < arrays.size(); k++) {
        void* p = arrays[k];
        const size_t bytes = sizes[k];
        buf.resize(bytes);
        if (bytes && std::fread(buf.data(), 1, bytes, f) != bytes) {
            std::fclose(f);
            return fail(c, GS3DC_ERR_INVALID_ARG, "%s is truncated", path);
        }
        if (bytes && cudaMemcpy(p, buf.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            std::fclose(f);
            return fail(c, GS3DC_ERR_CUDA, "upload of the training state failed");
        }
    }
    std::fclose(f);
    c->adam_step = h.adam_step;
    // the device's count of applied Adam steps follows the restored counter
    Persist ps{};
    ps.applied_steps = (unsigned long long)h.adam_step;
    CK(cudaMemcpy(c->persist, &ps, sizeof(Persist), cudaMemcpyHostToDevice));
    *c->persist_host = ps;
    // the FP32 model arrays mirror the restored reduced-storage model
    if (chosen_form(c) && (rc = unload_chosen(c))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
    return GS3DC_OK;
}


// ---- adaptive density control ----

// The controller's LCG advanced n steps on the host (s -> a s + c, mod 2^64).
static unsigned long long lcg_advance(unsigned long long s, unsigned long long n) {
    unsigned long long a = 6364136223846793005ULL, cc = 1442695040888963407ULL, ja = 1ULL, jc = 0ULL;
    while (n) {
        if (n & 1ULL) {
            ja = a * ja;
            jc = a * jc + cc;
        }
        cc = a * cc + cc;
        a = a * a;
        n >>= 1;
    }
    return ja * s + jc;
}

static DensityPtrs dc_ptrs(gs3dc_ctx* c) {
    return {c->dc_accum.p, c->dc_denom.p, c->dc_maxr.p, c->dc_clone.p, c->dc_split.p, c->dc_crank.p,
            c->dc_srank.p, c->dc_src.p, c->dc_keep.p, c->dc_out.p, c->dc_sums.p};
}

// DensityController::reset (density_controller.cpp:22-26): zeroed statistics for N.
static int dc_reset(gs3dc_ctx* c, int N) {
    const size_t n = N > 0 ? (size_t)N : 1;
    CK(c->dc_accum.ensure(n));
    CK(c->dc_denom.ensure(n));
    CK(c->dc_maxr.ensure(n));
    CK(cudaMemsetAsync(c->dc_accum.p, 0, n * 4, c->stream));
    CK(cudaMemsetAsync(c->dc_denom.p, 0, n * 4, c->stream));
    CK(cudaMemsetAsync(c->dc_maxr.p, 0, n * 4, c->stream));
    c->dc_n = N;
    return GS3DC_OK;
}

// Exclusive scan of n int flags into out; returns the total through *total (synchronises).
static int dc_scan(gs3dc_ctx* c, const int* in, int* out, int n, int* total) {
    const size_t nb = ((size_t)n + 1023) / 1024;
    CK(c->dc_sums.ensure(nb + 1));
    CK(cudaMemsetAsync(c->dc_sums.p, 0, (nb + 1) * 4, c->stream));
    CK(launch_scan_int(c->stream, in, out, c->dc_sums.p, n));
    CK(cudaMemcpyAsync(total, c->dc_sums.p + nb, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_raster_backward_lists(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg,
                                const float* d_image, float* d_means2D, float* d_conics, float* d_rgb,
                                float* d_opacities_2d, int64_t* list_bytes) {
    if (!c || !d_image) return GS3DC_ERR_INVALID_ARG;
    if (int rc_ = require_plain(c, "gs3dc_raster_backward_lists")) return rc_;
    int rc;
    if ((rc = check_config(c, cam, cfg))) return rc;
    if (!c->have_raster || c->screen_imported)
        return fail(c, GS3DC_ERR_STATE, "gs3dc_raster_backward_lists needs gs3dc_rasterize of the device model first");
    CK(cudaSetDevice(c->device));
    const size_t np = (size_t)c->W * c->H, n = (size_t)c->screen_n;
    if (np >= 0x7fffffffu) return fail(c, GS3DC_ERR_INVALID_ARG, "%zu pixels: the list offsets are 32-bit", np);
    CK(c->d_image.ensure(3 * np));
    CK(cudaMemcpyAsync(c->d_image.p, d_image, 3 * np * 4, cudaMemcpyHostToDevice, c->stream));
    if ((rc = push_params(c, cam, cfg, nullptr, 0, nullptr))) return rc;
    // entry offsets: exclusive scan of the forward's contributor counts
    CK(c->list_off.ensure(np + 1));
    int total = 0;
    if ((rc = dc_scan(c, c->n_contrib.p, c->list_off.p, (int)np, &total))) return rc;
    CK(c->lists.ensure(total > 0 ? (size_t)total : 1));
    CK(cudaMemsetAsync(c->dm2.p, 0, 2 * n * 4, c->stream));
    CK(cudaMemsetAsync(c->dcon.p, 0, 3 * n * 4, c->stream));
    CK(cudaMemsetAsync(c->drgb.p, 0, 3 * n * 4, c->stream));
    CK(cudaMemsetAsync(c->dop.p, 0, n * 4, c->stream));
    const int w = c->sorted_which;
    CK(launch_list_fill(c->stream, c->sp_dev, c->num_tiles, c->ranges.p, c->vals[w].p, screen_ptrs(c, false),
                        c->n_contrib.p, c->list_off.p, c->lists.p));
    CK(launch_list_bwd(c->stream, c->sp_dev, c->num_tiles, screen_ptrs(c, false), pixel_ptrs(c), c->list_off.p,
                       c->lists.p, rgrad_ptrs(c)));
    if ((rc = download(c, d_means2D, c->dm2.p, 2 * n * 4)) || (rc = download(c, d_conics, c->dcon.p, 3 * n * 4)) ||
        (rc = download(c, d_rgb, c->drgb.p, 3 * n * 4)) || (rc = download(c, d_opacities_2d, c->dop.p, n * 4)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    if (list_bytes) *list_bytes = (int64_t)(np * sizeof(int) + (size_t)total * sizeof(uint2));
    c->have_rgrad = true;
    return GS3DC_OK;
}

// The statistics pass of Trainer::step_with_densify (trainer.cpp:113-145): forward
// with the fused L1 and the raster backward of the current model, then the
// accumulation of |d_means2D| and the radii.  The target sits at gt_dev.
static int dc_stats_pass(gs3dc_ctx* c, const gs3d_camera* cam, const gs3d_render_config* cfg,
                  const gs3d_train_config* tc, int iteration, const float* gt_dev) {
    int rc;
    for (int attempt = 0; attempt < 3; attempt++) {
        if ((rc = push_params(c, cam, cfg, tc, iteration, gt_dev))) return rc;
        if ((rc = seq_train_front(c))) return rc;
        const int w = c->sorted_which;
        CK(launch_raster_fwd_plain(c->stream, c->sp_dev, c->num_tiles, true, c->ranges.p, c->tile_order.p,
                                   c->vals[w].p, screen_ptrs(c, false), pixel_ptrs(c), c->ctrl, c->fwd_ppt, c->fwd_batch));
        CK(launch_raster_bwd_plain(c->stream, c->sp_dev, c->num_tiles, true, c->ranges.p, c->tile_order.p,
                                   c->vals[w].p, screen_ptrs(c, false), pixel_ptrs(c), rgrad_ptrs(c), c->ctrl,
                                   c->bwd_ppt, c->bwd_batch));
        if ((rc = read_control(c))) return rc;
        if (c->persist_host->sticky_overflow) {
            if ((rc = acknowledge_overflow(c))) return rc;
            const unsigned long long P = c->ctrl_host->total_pairs;
            // the raster gradients of an overflowed pass are discarded
            const size_t n = (size_t)c->N;
            CK(cudaMemsetAsync(c->dm2.p, 0, 2 * n * 4, c->stream));
            CK(cudaMemsetAsync(c->dcon.p, 0, 3 * n * 4, c->stream));
            CK(cudaMemsetAsync(c->drgb.p, 0, 3 * n * 4, c->stream));
            CK(cudaMemsetAsync(c->dop.p, 0, n * 4, c->stream));
            if ((rc = ensure_pairs(c, P + P / 2 + 4096, c->num_tiles))) return rc;
            continue;
        }
        if (c->dc_n != c->N && (rc = dc_reset(c, c->N))) return rc;
        CK(launch_dc_accumulate(c->stream, c->N, c->dm2.p, c->radius.p, dc_ptrs(c), true));
        // the other raster-gradient accumulators start at zero for the next step
        const size_t n = (size_t)c->N;
        CK(cudaMemsetAsync(c->dcon.p, 0, 3 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->drgb.p, 0, 3 * n * 4, c->stream));
        CK(cudaMemsetAsync(c->dop.p, 0, n * 4, c->stream));
        c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = false;
        return GS3DC_OK;
    }
    return fail(c, GS3DC_ERR_PAIR_OVERFLOW, "tile-pair capacity kept overflowing in the statistics pass");
}

int gs3dc_density_accumulate(gs3dc_ctx* c, const float* d_means2D, const int* radii) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    int rc;
    if ((rc = require_model(c)) || (rc = require_plain(c, "density control"))) return rc;
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->N;
    if (c->dc_n != c->N && (rc = dc_reset(c, c->N))) return rc;
    if (n == 0) return GS3DC_OK;
    float* dm = nullptr;
    const int* rd = nullptr;
    if (d_means2D) {
        CK(c->dc_dm_in.ensure(2 * n));
        CK(cudaMemcpyAsync(c->dc_dm_in.p, d_means2D, 2 * n * 4, cudaMemcpyHostToDevice, c->stream));
        dm = c->dc_dm_in.p;
        if (radii) {
            CK(c->dc_radii_in.ensure(n));
            CK(cudaMemcpyAsync(c->dc_radii_in.p, radii, n * 4, cudaMemcpyHostToDevice, c->stream));
            rd = c->dc_radii_in.p;
        }
    } else {
        if (!c->have_rgrad)
            return fail(c, GS3DC_ERR_STATE, "gs3dc_density_accumulate(NULL) needs gs3dc_raster_backward first");
        dm = c->dm2.p;
        rd = c->radius.p;
    }
    CK(launch_dc_accumulate(c->stream, c->N, dm, rd, dc_ptrs(c), false));
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_densify_and_prune(gs3dc_ctx* c, const gs3d_densify_config* dcfg, float scene_extent, int* new_count) {
    if (!c || !dcfg) return GS3DC_ERR_INVALID_ARG;
    int rc;
    if ((rc = require_model(c)) || (rc = require_plain(c, "density control"))) return rc;
    if (!c->model_raw) return fail(c, GS3DC_ERR_STATE, "density control needs a raw model (gs3dc_set_raw_params)");
    CK(cudaSetDevice(c->device));
    if ((rc = gs3dc_synchronize(c))) return rc;
    const int N = c->N;
    if (N == 0) {
        if (new_count) *new_count = 0;
        return GS3DC_OK;
    }
    if (c->dc_n != N && (rc = dc_reset(c, N))) return rc;   // no statistics: every average is zero
    const size_t n = (size_t)N;
    const int mc3 = c->max_coeffs * 3;
    CK(c->dc_clone.ensure(n));
    CK(c->dc_split.ensure(n));
    CK(c->dc_crank.ensure(n));
    CK(c->dc_srank.ensure(n));
    // clone / split classes and their ranks (density_controller.cpp:45-124)
    const float size_thr = 0.01f * scene_extent;
    CK(launch_dc_classify(c->stream, N, c->sc.p, dc_ptrs(c), dcfg->grad_threshold, size_thr));
    int n_c = 0, n_s = 0;
    if ((rc = dc_scan(c, c->dc_clone.p, c->dc_crank.p, N, &n_c)) ||
        (rc = dc_scan(c, c->dc_split.p, c->dc_srank.p, N, &n_s)))
        return rc;
    const int M = N + n_c + n_s;
    const size_t m = (size_t)M;
    CK(c->dc_src.ensure(m));
    CK(c->dc_keep.ensure(m));
    CK(c->dc_out.ensure(m));
    const size_t widths[5] = {3, 3, 4, (size_t)mc3, 1};
    for (int k = 0; k < 5; k++) CK(c->dc_t[k].ensure(widths[k] * m));
    const ModelPtrs t{c->dc_t[0].p, c->dc_t[1].p, c->dc_t[2].p, c->dc_t[3].p, c->dc_t[4].p};
    const float log_factor = std::log(0.8f * 2.0f);   // density_controller.cpp:105, the reference's libm
    CK(launch_dc_expand(c->stream, N, n_c, n_s, model_ptrs(c), mc3, dc_ptrs(c), t, c->dc_rng, log_factor));
    // prune (density_controller.cpp:144-170) and compact
    CK(launch_dc_keep(c->stream, M, N, t, dc_ptrs(c), dcfg->min_opacity, dcfg->max_screen_size,
                      0.1f * scene_extent));
    int kept = 0;
    if ((rc = dc_scan(c, c->dc_keep.p, c->dc_out.p, M, &kept))) return rc;
    const size_t nn = kept > 0 ? (size_t)kept : 1;
    for (int k = 0; k < 5; k++) CK(c->dc_new[k].ensure(widths[k] * nn));
    const ModelPtrs o{c->dc_new[0].p, c->dc_new[1].p, c->dc_new[2].p, c->dc_new[3].p, c->dc_new[4].p};
    CK(launch_dc_compact(c->stream, M, kept, t, mc3, dc_ptrs(c), o));
    CK(cudaStreamSynchronize(c->stream));
    c->dc_rng = lcg_advance(c->dc_rng, 12ull * (unsigned long long)n_s);
    // the new model replaces the old arrays
    std::swap(c->pos.p, c->dc_new[0].p);
    std::swap(c->pos.n, c->dc_new[0].n);
    std::swap(c->sc.p, c->dc_new[1].p);
    std::swap(c->sc.n, c->dc_new[1].n);
    std::swap(c->rot.p, c->dc_new[2].p);
    std::swap(c->rot.n, c->dc_new[2].n);
    std::swap(c->sh.p, c->dc_new[3].p);
    std::swap(c->sh.n, c->dc_new[3].n);
    std::swap(c->op.p, c->dc_new[4].p);
    std::swap(c->op.n, c->dc_new[4].n);
    drop_graphs(c);
    if ((rc = ensure_model(c, kept, c->max_coeffs))) return rc;
    c->N = kept;
    const size_t kn = (size_t)kept;
    if (kn) {   // raster-gradient accumulators start at zero
        CK(cudaMemsetAsync(c->dm2.p, 0, 2 * kn * 4, c->stream));
        CK(cudaMemsetAsync(c->dcon.p, 0, 3 * kn * 4, c->stream));
        CK(cudaMemsetAsync(c->drgb.p, 0, 3 * kn * 4, c->stream));
        CK(cudaMemsetAsync(c->dop.p, 0, kn * 4, c->stream));
    }
    if ((rc = dc_reset(c, kept))) return rc;
    // Trainer::step_with_densify resets the optimiser when the count changed (trainer.cpp:157-161)
    if (kept != N && ((rc = ensure_adam(c)) || (rc = zero_adam(c)))) return rc;
    c->have_screen = c->have_pairs = c->have_sorted = c->have_raster = c->have_rgrad = c->have_grads = false;
    c->have_step_grads = false;
    CK(cudaStreamSynchronize(c->stream));
    if (new_count) *new_count = kept;
    return GS3DC_OK;
}

int gs3dc_reset_opacity(gs3dc_ctx* c) {
    if (!c) return GS3DC_ERR_INVALID_ARG;
    int rc;
    if ((rc = require_model(c)) || (rc = require_plain(c, "density control"))) return rc;
    if (!c->model_raw) return fail(c, GS3DC_ERR_STATE, "gs3dc_reset_opacity needs a raw model");
    CK(cudaSetDevice(c->device));
    // inverse_sigmoid(0.01) with the reference's libm (density_controller.cpp:198)
    CK(launch_fill(c->stream, c->op.p, c->N, std::log(0.01f / 0.99f)));
    CK(cudaStreamSynchronize(c->stream));
    return GS3DC_OK;
}

int gs3dc_train_step_densify(gs3dc_ctx* c, const gs3d_camera* cam, const float* gt, int gt_on_device,
                             const gs3d_render_config* cfg, const gs3d_train_config* tc,
                             const gs3d_densify_config* dcfg, float scene_extent, int iteration, float* loss,
                             int* n_gaussians) {
    if (!c || !gt || !tc || !dcfg) return GS3DC_ERR_INVALID_ARG;
    int rc;
    if ((rc = check_config(c, cam, cfg)) || (rc = require_model(c)) ||
        (rc = require_plain(c, "gs3dc_train_step_densify")))
        return rc;
    CK(cudaSetDevice(c->device));
    const float* gt_dev = gt;
    if (!gt_on_device) {   // one device copy serves the step and the statistics pass
        const size_t np = (size_t)cam->width * cam->height;
        CK(c->gt.ensure(3 * np));
        CK(cudaMemcpyAsync(c->gt.p, gt, 3 * np * 4, cudaMemcpyHostToDevice, c->stream));
        gt_dev = c->gt.p;
    }
    float l = 0.0f;
    if ((rc = gs3dc_train_step(c, cam, gt_dev, 1, cfg, tc, iteration, &l))) return rc;
    if ((rc = dc_stats_pass(c, cam, cfg, tc, iteration, gt_dev))) return rc;
    if (dcfg->enabled && iteration >= dcfg->densify_from_iter && iteration < dcfg->densify_until_iter &&
        dcfg->densify_interval > 0 && iteration % dcfg->densify_interval == 0) {
        if ((rc = gs3dc_densify_and_prune(c, dcfg, scene_extent, nullptr))) return rc;
    }
    if (dcfg->enabled && dcfg->opacity_reset_interval > 0 && iteration > 0 &&
        iteration % dcfg->opacity_reset_interval == 0) {
        if ((rc = gs3dc_reset_opacity(c))) return rc;
    }
    CK(cudaStreamSynchronize(c->stream));
    if (loss) *loss = l;
    if (n_gaussians) *n_gaussians = c->N;
    return GS3DC_OK;
}
}  // extern "C"
