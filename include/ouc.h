/*
 * ouc.h -- C ABI of the B200-native elastic P/S-decoupled finite-difference
 * modeling and reverse-time-migration library (libouc.so).
 *
 * The reference (gm340/ouc, P-S-seperating.cu) has no library API: its
 * interface is a set of __global__ kernels driven by a monolithic main().
 * Each entry point below replaces one stage of that main(); the comment on
 * each names the reference lines whose role it takes over.  "PS:n" means
 * P-S-seperating.cu line n.
 *
 * Conventions
 *   - Every call returns an int status: OUC_OK (0) or an OUC_E* code; no
 *     exception or abort crosses the ABI.  ouc_last_error() gives the detail.
 *   - Grids are x-major with z contiguous: element (i, j) of an nx x nz
 *     array is a[i * nz + j] (the reference's i * Zn + j, PS:224).
 *   - "Padded" coordinates include the absorbing layer of npml cells on
 *     every side (X = nx + 2 npml, Z = nz + 2 npml); source and receiver
 *     positions in ouc_shot are interior coordinates (padded - npml).
 *   - The caller owns host buffers; the library owns device buffers.  The
 *     *_dev entry points take device pointers instead and do no host copy.
 *   - A context is not thread-safe; use one context per host thread.  All
 *     work is queued on the context's stream.
 */
#ifndef OUC_H
#define OUC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OUC_VERSION_MAJOR 0
#define OUC_VERSION_MINOR 1

enum {
    OUC_OK = 0,
    OUC_EINVAL = 1,      /* bad argument or configuration                      */
    OUC_ECUDA = 2,       /* a CUDA runtime call failed                          */
    OUC_ENOMEM = 3,      /* device allocation failed                            */
    OUC_EUNSTABLE = 4,   /* CFL limit exceeded or non-finite wavefield          */
    OUC_ESTATE = 5,      /* call out of order (e.g. stack before any shot)      */
    OUC_ETIMEOUT = 6,    /* a bounded device wait ran out                       */
    OUC_ENODEV = 7,      /* no usable sm_100 device                             */
    OUC_ESCRATCH = 8     /* problem larger than the fixed scratch of ouc_forward_noalloc */
};

enum { OUC_MODEL_INTERIOR = 0, OUC_MODEL_PADDED = 1 };
/* Which time level the Vx/Vz boundary strips are restored at during the
 * source-wavefield reconstruction.  REFERENCE reproduces PS:2337 (one level
 * late, as the reference does); EXACT restores the level the inverse
 * leapfrog needs, which reconstructs the source field to round-off. */
enum { OUC_STRIP_REFERENCE = 0, OUC_STRIP_EXACT = 1 };
/* Which source level the imaging condition correlates at back-step t:
 * REFERENCE = the level the reference uses (PS:964, PS:2361), EXACT = the
 * level whose records were injected at that step. */
enum { OUC_IMAGE_REFERENCE = 0, OUC_IMAGE_EXACT = 1 };
enum { OUC_PREC_FP32 = 0, OUC_PREC_FP16 = 1, OUC_PREC_BF16 = 2 };
/* Source mechanism: THETA adds the wavelet to the dilatation stress at the
 * source cell (PS:331-338, PS:380); FORCE_Z adds dt^2 * wavelet to the
 * vertical P displacement (an extension with no reference counterpart). */
enum { OUC_SRC_THETA = 0, OUC_SRC_FORCE_Z = 1 };
/* Gather layout at the host boundary: receiver-major [X][nt] as the
 * reference's record arrays (PS:308), or time-major [nt][X]. */
enum { OUC_GATHER_XT = 0, OUC_GATHER_TX = 1 };

typedef struct ouc_config {
    int nx, nz;             /* interior grid                                     */
    int npml;               /* absorbing width L in cells (PS:15)                */
    int half_order;         /* stencil half-width N: 2, 5 or 6 (PS:16 uses 6)    */
    float dx, dz, dt;       /* spacing (m) and time step (s)                     */
    int nt;                 /* time steps per shot (PS:17)                       */
    double pml_r;           /* target reflection R of the damping profile (PS:23)  */
    int model_layout;       /* OUC_MODEL_INTERIOR or OUC_MODEL_PADDED            */
    int strip_level;        /* OUC_STRIP_*                                       */
    int image_align;        /* OUC_IMAGE_*                                       */
    int strip_precision;    /* OUC_PREC_*: storage of the saved source wavefield
                               (boundary strips, or the snapshots below); FP16 is
                               scaled by a power of two per slot and field      */
    int compensated_image;  /* 1: compensated-FP32 per-shot accumulators         */
    int gather_layout;      /* OUC_GATHER_*                                      */
    int device;             /* CUDA device ordinal                               */
    void* stream;           /* cudaStream_t to run on, or NULL for a private one */
    int max_batch;          /* shots advanced together per launch (0 or 1: one)  */
    int snapshot_every;     /* 0: rebuild the source wavefield backwards from the
                               boundary strips (the reference's method, PS:2326-
                               2361); K >= 1: store the source P wavefield of
                               every K-th imaging level during the forward pass
                               and image only those levels (no reconstruction;
                               no counterpart in the reference)                 */
    int density;            /* 1: variable density from the rho model (moduli
                               rho Vp^2, rho Vs^2; acceleration = buoyancy x
                               stress divergence, buoyancy averaged onto the
                               staggered Ux/Uz positions); 0: the reference's
                               density-normalised equations, rho ignored (no
                               counterpart in the reference for 1)             */
    int gradient;           /* 1: RTM shots also accumulate the FWI gradient
                               (ouc_gradient; strip form, density = 0)        */
    int use_graphs;         /* 1: capture each whole-shot time loop (one launch
                               per stage and step) as a CUDA graph on first use
                               and replay it for later shots and batches        */
} ouc_config;

typedef struct ouc_shot {
    int sx, sz;             /* source cell, interior coordinates                 */
    int rz;                 /* receiver row, interior z (receivers span all X)   */
    int src_type;           /* OUC_SRC_*                                         */
    int t0;                 /* wavelet delay in samples, for the mute (PS:1955)  */
    int mute;               /* 1: direct-wave mute before back-propagation       */
} ouc_shot;

typedef struct ouc_ctx ouc_ctx;

/* Per-call device timings (CUDA events on the context stream), ms. */
typedef struct ouc_timing {
    float forward_ms;       /* forward time loop                                 */
    float backward_ms;      /* backward time loop incl. imaging                  */
    float finalize_ms;      /* image normalisation, Laplacian, stack             */
    float copy_ms;          /* host<->device copies inside the call              */
    long long kernel_launches;
} ouc_timing;

const char* ouc_strerror(int status);
const char* ouc_last_error(const ouc_ctx* ctx);
int ouc_version(void);

/* Float32 staggered-grid weights a_1..a_N the library uses (PS:221 for N=6,
 * the exact Taylor solution rounded to float32 otherwise). */
int ouc_stencil_weights(int half_order, float* out);

/* Ricker wavelet as built by main() (PS:1954-1958): out[nt], *t0 = delay. */
int ouc_ricker(float fm, float dt, int nt, float* out, int* t0);

/* Create a context: uploads the model, pads it into the absorbing layer
 * (xiangbian, PS:37-119), builds the damping profile (PS:2067-2105) and
 * allocates all device state.  vp/vs/rho are nx*nz (OUC_MODEL_INTERIOR) or
 * X*Z (OUC_MODEL_PADDED); rho may be NULL and is not used by the
 * reference's density-normalised equations (PS:373-378) unless cfg->density. */
int ouc_create(const ouc_config* cfg, const float* vp, const float* vs, const float* rho, ouc_ctx** out);
int ouc_destroy(ouc_ctx* ctx);
int ouc_dims(const ouc_ctx* ctx, int* X, int* Z);
void* ouc_stream(const ouc_ctx* ctx);
int ouc_last_timing(const ouc_ctx* ctx, ouc_timing* t);
/* Device bytes held by the context (state, strips, staging). */
size_t ouc_device_bytes(const ouc_ctx* ctx);

/* Forward modeling of one shot: the reference's forward time loop
 * (forward_s + forward_u, PS:2258-2266) with receiver extraction (PS:307-311,
 * post-update values).  gather_vx/vz: X*nt each in cfg->gather_layout, or
 * NULL.  fields: optional 6*X*Z output of the final Ux Uz Px Pz Sx Sz. */
int ouc_forward(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, float* gather_vx, float* gather_vz,
                float* fields);
int ouc_forward_dev(ouc_ctx* ctx, const ouc_shot* shot, const float* d_wavelet, float* d_gather_vx,
                    float* d_gather_vz);

/* Forward modeling with the first-order velocity-stress scheme of the
 * reference's stress (PS:487-560) and velocity (PS:390-486) kernels, which
 * its main() never calls: split stresses theta_x/z, omega_x/z and the four Q
 * fields with the split-field damping (1 - dt a/2)/(1 + dt a/2) of the
 * context's profile, the wavelet added to theta at the source cell, P/S
 * velocities updated from the stress derivatives, U = P + S recorded at the
 * receiver row after the update (the receiver test as a comparison,
 * PS:481).  Half-order 6 uses the kernels' own five-digit weights, other
 * orders the context's.  Theta source only; density-normalised contexts
 * only.  gather_vx/vz: X*nt each in cfg->gather_layout, or NULL.  fields:
 * optional 16*X*Z output of the final Vx Vz Vpx Vpz Vsx Vsz theta omega
 * duzdx duzdz duxdx duxdz theta_x theta_z omega_x omega_z. */
int ouc_forward_fo(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, float* gather_vx, float* gather_vz,
                   float* fields);
/* Receiver back-propagation with the same first-order scheme: the
 * reference's stress_backward_propagation (PS:821-887) and
 * velocity_backward_propagation (PS:728-820), i.e. the updates above without
 * source and record, for t = nt-1 .. 0, each step preceded by the records of
 * time t written into U at the receiver row on the interior columns [L, X-L)
 * (load_record, PS:1472-1481, as the launched receiver path orders it,
 * PS:2319).  rec_vx/rec_vz: X*nt each in cfg->gather_layout.  fields: as
 * ouc_forward_fo (theta without a source term). */
int ouc_backward_fo(ouc_ctx* ctx, const ouc_shot* shot, const float* rec_vx, const float* rec_vz, float* fields);

/* One RTM shot: forward with boundary-strip save (PS:2258-2292), optional
 * mute (PS:2293), receiver back-propagation with record injection and the
 * source-wavefield reconstruction (PS:2313-2364), PP/PS imaging (PS:2361),
 * normalisation and Laplacian (PS:2367-2373).  rec_vx/rec_vz are the
 * observed records (X*nt, cfg->gather_layout); NULL uses the records the
 * forward pass produces, as the reference's main() does.  img_pp/img_ps
 * receive the nx*nz Laplacian-filtered images (the per-shot files of
 * PS:2379-2400); either may be NULL.  The images are also added into the
 * context's FP64 stack. */
int ouc_rtm_shot(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, const float* rec_vx,
                 const float* rec_vz, float* img_pp, float* img_ps);
int ouc_rtm_shot_dev(ouc_ctx* ctx, const ouc_shot* shot, const float* d_wavelet, const float* d_rec_vx,
                     const float* d_rec_vz, float* d_img_pp, float* d_img_ps);

/* A batch of RTM shots on the same model, advanced together: every time
 * step of up to cfg->max_batch shots is one launch per stage (the reference
 * runs its shots one after another, PS:2108).  Per-shot arrays of pointers;
 * rec_vx/rec_vz may be NULL (self-modelled records for every shot) and any
 * img_* entry or array may be NULL.  All images enter the FP64 stack. */
int ouc_rtm_batch(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const float* wavelet,
                  const float* const* rec_vx, const float* const* rec_vz, float* const* img_pp,
                  float* const* img_ps);
int ouc_rtm_batch_dev(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const float* d_wavelet,
                      const float* const* d_rec_vx, const float* const* d_rec_vz, float* const* d_img_pp,
                      float* const* d_img_ps);

/* FP64 cross-shot stack of the Laplacian images (replaces the host FP32 sum
 * through per-shot files, PS:2403-2443) and the FP64 stacked illumination.
 * Any output may be NULL; reset != 0 clears the stack after reading. */
int ouc_stack(ouc_ctx* ctx, double* stack_pp, double* stack_ps, double* illum, int reset);
int ouc_stack_dev(ouc_ctx* ctx, const double** d_pp, const double** d_ps, const double** d_illum);

/* FWI gradient (cfg.gradient = 1; the step after imaging: the formula of the
 * reference's gradfun/caculate_Grad, PS:1518-1633, which its main() never
 * calls).  At every back-step of an RTM shot, with U_s = P + S the source
 * displacement at the level the imaging condition correlates there and the
 * receiver's stress fields (theta, omega, Q, PS:373-378) recomputed from its
 * displacement after the step, on the interior cells at least N from the
 * absorbing layers:
 *   G_vp -= 2 rho Vp (dUx/dx + dUz/dz) theta_r
 *   G_vs -= 2 rho Vs (omega_r (dUx/dz - dUz/dx) + Qzx_r dUz/dx + Qzz_r dUz/dz
 *                     + Qxz_r dUx/dz + Qxx_r dUx/dx)
 *   illum += Ux_s^2 + Uz_s^2
 * (rho from ouc_create's rho model, 1 without one; the reference's dUx/dz
 * stencil typo, PS:1556, is not reproduced).  Shots add into FP64 stacks in
 * order; ouc_gradient reads them (nx*nz each, any may be NULL), reset != 0
 * clears them. */
int ouc_gradient(ouc_ctx* ctx, double* g_vp, double* g_vs, double* illum, int reset);

/* Step-level interface: one RTM shot advanced one reference time step per
 * call, for comparing against the reference's kernels step by step.  The
 * calls must come in the order of the reference's main():
 *   ouc_step_begin                once: zero both wavefields and the imaging
 *                                 accumulators, take the wavelet and, if
 *                                 given, the observed records (host arrays,
 *                                 cfg.gather_layout; NULL: the forward steps
 *                                 record them, PS:307-311);
 *   ouc_step_forward(t)           t = 0 .. nt-1: forward_s + forward_u +
 *                                 record + save_wavefiled (PS:2261-2266); the
 *                                 last one also mutes the records when the
 *                                 shot asks for it (PS:2296-2297);
 *   ouc_step_receiver(t)          t = nt-1 .. 0: load_record + rt_s_res +
 *                                 rt_u_res (PS:2319-2324, 2349-2354);
 *   ouc_step_reconstruct(t)       after ouc_step_receiver(t): reshot_u,
 *                                 read_wavefiled1, reshot_s, read_wavefiled2
 *                                 and corr_v (PS:2326-2361);
 *   ouc_image_finalize            image_fun + Laplace (PS:2365-2376) into
 *                                 img_pp / img_ps (host, nx*nz, may be NULL),
 *                                 and the FP64 stack.
 * A call out of this order returns OUC_ESTATE and changes nothing.  Results
 * equal ouc_rtm_shot's bit for bit.  A whole-shot call (ouc_forward*,
 * ouc_rtm_*) ends a stepped shot.  ouc_step_fields copies the current
 * displacement of one wavefield (side 0 = source, 1 = receiver) to the host
 * as 6 padded X*Z arrays: Ux, Uz, Px, Pz, Sx, Sz (PS:291-303); during the
 * backward steps the source side holds the reconstructed wavefield, which
 * is defined on the interior only. */
int ouc_step_begin(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, const float* rec_vx,
                   const float* rec_vz);
int ouc_step_forward(ouc_ctx* ctx, int t);
int ouc_step_receiver(ouc_ctx* ctx, int t);
int ouc_step_reconstruct(ouc_ctx* ctx, int t);
int ouc_image_finalize(ouc_ctx* ctx, float* img_pp, float* img_ps);
int ouc_step_fields(ouc_ctx* ctx, int side, float* fields);

/* Survey on per-shot sub-grids (the batching form, no counterpart in the
 * reference, which runs every shot on the whole grid, PS:2108).  Each shot k
 * has an aperture: the interior columns [x0, x1) of the context's model that
 * its sub-grid covers (its source column inside).  The sub-grid is the
 * model's padded grid restricted to padded rows [x0, x1 + 2 npml): the
 * absorbing cells on either side hold the model itself, and the damping
 * profile is that of the sub-grid's own edges, so each shot equals a
 * single-shot run of a context created on that window as a padded model.
 * Shots are taken in the order given, up to cfg.max_batch per batch; the
 * shots of a batch may differ in width and advance together (one launch per
 * stage and time step, each CTA reading its shot's geometry).  Shot
 * coordinates are interior coordinates of the whole model.
 *   ouc_survey_forward: gathers per shot, (x1 - x0 + 2 npml) x nt each in
 *     cfg.gather_layout (host; any pointer may be NULL).
 *   ouc_survey_rtm: RTM of every shot (strip form only: snapshot_every = 0);
 *     rec_vx/rec_vz as the forward gathers or NULL (self-modelled); images
 *     (x1 - x0) x nz per shot (host, may be NULL); every image also enters
 *     the context's FP64 stack at rows [x0, x1), shot by shot in order. */
typedef struct ouc_aperture {
    int x0, x1;             /* interior columns [x0, x1) of the model           */
} ouc_aperture;
int ouc_survey_forward(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const ouc_aperture* apertures,
                       const float* wavelet, float* const* gather_vx, float* const* gather_vz);
int ouc_survey_rtm(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const ouc_aperture* apertures,
                   const float* wavelet, const float* const* rec_vx, const float* const* rec_vz, float* const* img_pp,
                   float* const* img_ps);

/* Autotuner of the launch batch (no counterpart in the reference): times
 * `steps` forward steps of 1, 2, 4, ... and cfg.max_batch shots per launch on
 * this context's grid (CUDA events; the wavelet buffer is cleared) and keeps
 * the batch with the fewest ns per cell-update (a larger batch must be 3 %
 * faster to win); *best_batch and *ns_per_cell may be NULL.  Later
 * ouc_rtm_batch / ouc_survey_* calls advance that many shots per launch.
 * ouc_set_run_batch sets it directly (1 .. cfg.max_batch), e.g. from a cache
 * of earlier tuning results.  It keeps the current step-kernel geometry;
 * ouc_tune below chooses both. */
int ouc_tune_batch(ouc_ctx* ctx, int steps, int* best_batch, float* ns_per_cell);
int ouc_set_run_batch(ouc_ctx* ctx, int n);
/* Joint tuning of the launch batch and the step-kernel geometry: for each
 * batch candidate, forward steps are timed with the tile kernel and with the
 * x-marching kernel at segment lengths 64 .. 512 rows; the fastest geometry
 * per batch is kept and the batch is chosen as ouc_tune_batch does.  Both
 * choices are applied to the context; each output pointer may be NULL. */
int ouc_tune(ouc_ctx* ctx, int steps, int* best_batch, int* best_seg_rows, float* ns_per_cell);

/* Step-kernel geometry.  seg_rows > 0 (a multiple of 16): the x-marching
 * kernel, each CTA walking a 64-column strip down a segment of that many rows
 * in 16-row blocks with bulk asynchronous row copies; 0: one CTA per 32 x 64
 * tile; OUC_STEP_TILE_QUEUE: the tile kernel as a persistent launch (two
 * CTAs per SM) claiming (tile, shot) items from a dynamic queue, heaviest
 * tiles (damping layers, boundary ring) first.  All replace the reference's per-step kernel pair (forward_s +
 * forward_u, PS:316-384 / PS:205-314, and their receiver and reconstruction
 * twins) with bit-identical results.  ouc_create picks the tile kernel;
 * ouc_tune times both geometries.  Changing it drops the captured time
 * loops (they are captured again on next use). */
#define OUC_STEP_TILE_QUEUE (-1)
int ouc_set_step_kernel(ouc_ctx* ctx, int seg_rows);
int ouc_get_step_kernel(const ouc_ctx* ctx, int* seg_rows);

/* Test hook for the step kernels' bounded copy wait (no counterpart in the
 * reference).  on = 1: every tile of the tile kernels expects 16 bytes more
 * than its tensor copies deliver, so each CTA's wait on them runs out (about
 * 40 ms), records the failure and leaves its tile unwritten; the next
 * whole-shot call returns OUC_ETIMEOUT and clears the record.  on = 0 (the
 * default) restores normal operation; the context stays usable.  Drops the
 * captured time loops. */
int ouc_debug_copy_stall(ouc_ctx* ctx, int on);

/* Device time of one launch of each step kernel at batch n (ms[0] forward,
 * ms[1] receiver, ms[2] reconstruction + imaging), averaged over `reps`
 * launches after one warm-up, on the state the last RTM batch of n shots
 * left (call it right after such a batch; the state is consumed).  CUDA
 * events on the context stream. */
int ouc_time_step_kernels(ouc_ctx* ctx, int n, int reps, float* ms);

/* Forward modeling that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot allocate device memory when they need
 * a modeling run: applications whose own memory pool owns the whole GPU and
 * forbids other allocations, and pipelines that reserve memory up front and
 * must not enter the allocator later (cudaMalloc/cudaFree synchronise the
 * device and can fail under memory pressure).  Same kernels and results as
 * ouc_forward; the wavefield state lives in a fixed library-owned device
 * array of OUC_NOALLOC_SCRATCH_BYTES (held on each GPU that loads it until
 * process exit).  Inputs and outputs are the caller's device buffers:
 * d_vp, d_vs padded X*Z models (x-major), d_wavelet nt samples, gathers X*nt
 * each in cfg->gather_layout.  cfg->model_layout must be OUC_MODEL_PADDED and
 * cfg->density 0 (density-normalised equations only); other values return
 * OUC_EINVAL before any device work.  A CUDA error already pending on the
 * calling thread returns OUC_ECUDA and is left for its owner to read.  Work
 * is queued on cfg->stream and the call
 * returns without synchronising.  The first call on a device looks up the
 * array's address and sets the kernels' shared-memory limit there: make it
 * before any stream capture on that device.  All
 * calls share the array and it keeps the last call's contents (each call
 * clears what it needs zeroed); calls whose work overlaps on the GPU race, so
 * serialise them.  Sizes beyond the array return OUC_ESCRATCH; the CFL check
 * of ouc_create is the caller's responsibility here. */
#define OUC_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int ouc_forward_noalloc(const ouc_config* cfg, const ouc_shot* shot, const float* d_vp, const float* d_vs,
                        const float* d_wavelet, float* d_gather_vx, float* d_gather_vz);

#ifdef __cplusplus
}
#endif
#endif /* OUC_H */
