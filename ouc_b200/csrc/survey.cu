// Survey of many shots on per-shot sub-grids of one model (the batching
// form): each shot runs on a window of the model around its aperture, and a
// batch of up to cfg.max_batch shots of different widths advances together,
// one launch per stage and time step.  blockIdx.y selects the shot and the
// CTA reads that shot's grid geometry (width, ring, model window) from its
// descriptor; CTAs beyond a narrower shot's width exit at once, so one launch
// covers uneven shots with no host-side splitting.
//
// A shot's sub-grid is the model's padded grid restricted to the rows
// [x0, x1 + 2 npml) (interior columns [x0, x1) plus the absorbing cells on
// either side, which hold the model itself rather than edge copies), with the
// damping profile of its own edges.  Each shot's result equals a single-shot
// run on that window given as a padded model (checked in the GPU tests).
// Images are (x1 - x0) x nz and enter the context's FP64 stack at rows
// [x0, x1), shot by shot in order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ouc.h"
#include "ctx.h"

namespace ouc {
namespace survey {

using namespace host;

#define CKS(call)                                                          \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) return host::cuda_fail(ctx, e_, #call);     \
    } while (0)

constexpr int kModelFields = 6;   // vp2 vs2 ax az bx bz per batch slot

float* slot_field(const ouc_ctx* c, int b, int k) {
    return c->sv_model + ((size_t)b * kModelFields + k) * c->fstride + (size_t)kGX * c->pitch + kZOFF;
}

int ensure_model(ouc_ctx* ctx) {
    if (ctx->sv_model) return OUC_OK;
    const size_t bytes = (size_t)ctx->batch * kModelFields * ctx->fstride * sizeof(float);
    if (cudaMalloc(&ctx->sv_model, bytes) != cudaSuccess) {
        cudaGetLastError();
        ctx->sv_model = nullptr;
        return fail(ctx, OUC_ENOMEM, "cannot allocate the sub-grid models");
    }
    ctx->bytes += bytes;
    return OUC_OK;
}

struct Window {
    int x0, X;   // first padded row in the model's grid, padded width
};

int check(ouc_ctx* ctx, int n, const ouc_shot* shots, const ouc_aperture* ap) {
    if (n < 1 || !shots || !ap) return fail(ctx, OUC_EINVAL, "no shots or apertures");
    if (ctx->cfg.snapshot_every > 0) return fail(ctx, OUC_EINVAL, "the survey runs the strip form (snapshot_every = 0)");
    if (ctx->cfg.gradient) return fail(ctx, OUC_EINVAL, "the survey does not compute the FWI gradient");
    for (int k = 0; k < n; ++k) {
        int rc = check_shot(ctx, &shots[k]);
        if (rc) return rc;
        const int x0 = ap[k].x0, x1 = ap[k].x1;
        if (x0 < 0 || x1 > ctx->nx || x1 - x0 < 4 * ctx->N)
            return fail(ctx, OUC_EINVAL, "aperture outside the model or narrower than 4N");
        if (shots[k].sx < x0 || shots[k].sx >= x1) return fail(ctx, OUC_EINVAL, "source outside its aperture");
    }
    return OUC_OK;
}

// Descriptors and sub-grid models of one batch; `keep` holds the host
// damping arrays until the batch's final synchronisation.
int upload_batch(ouc_ctx* ctx, int n, const ouc_shot* shots, const ouc_aperture* ap, const float* d_w,
                 std::vector<std::vector<float>>& keep) {
    int rc = ensure_model(ctx);
    if (rc) return rc;
    const int L = ctx->L, Z = ctx->Z, TX = 32, pitch = ctx->pitch;
    CKS(cudaMemsetAsync(ctx->sv_model, 0, (size_t)n * kModelFields * ctx->fstride * sizeof(float), ctx->stream));
    std::vector<ShotDesc> d(n);
    for (int b = 0; b < n; ++b) {
        const Window w{ap[b].x0, ap[b].x1 - ap[b].x0 + 2 * L};
        // model window: rows [x0, x0 + X) of the padded model, guard columns included
        const float* window_src[kModelFields] = {ctx->vp2, ctx->vs2, nullptr, nullptr, ctx->bx, ctx->bz};
        for (int k = 0; k < kModelFields; ++k) {
            if (!window_src[k] || (k >= 4 && !ctx->cfg.density)) continue;
            const float* src = window_src[k] - kZOFF + (size_t)w.x0 * pitch;
            CKS(cudaMemcpyAsync(slot_field(ctx, b, k) - kZOFF, src, (size_t)w.X * pitch * sizeof(float),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        }
        // damping profile of the window's own edges (the profile a context
        // created on this window as a padded model computes)
        std::vector<float> vpw(ctx->vp_host.begin() + (size_t)w.x0 * Z, ctx->vp_host.begin() + (size_t)(w.x0 + w.X) * Z);
        keep.emplace_back((size_t)w.X * Z);
        keep.emplace_back((size_t)w.X * Z);
        std::vector<float>& ax = keep[keep.size() - 2];
        std::vector<float>& az = keep[keep.size() - 1];
        damping(vpw, w.X, Z, L, ctx->cfg.pml_r, ax, az);
        CKS(cudaMemcpy2DAsync(slot_field(ctx, b, 2), (size_t)pitch * 4, ax.data(), (size_t)Z * 4, (size_t)Z * 4, w.X,
                              cudaMemcpyHostToDevice, ctx->stream));
        CKS(cudaMemcpy2DAsync(slot_field(ctx, b, 3), (size_t)pitch * 4, az.data(), (size_t)Z * 4, (size_t)Z * 4, w.X,
                              cudaMemcpyHostToDevice, ctx->stream));
        ShotDesc& s = d[b];
        memset(&s, 0, sizeof(s));
        s.sx = shots[b].sx - w.x0 + L;
        s.sz = shots[b].sz + L;
        s.rz = shots[b].rz + L;
        s.src_type = shots[b].src_type;
        s.wavelet = d_w;
        s.gather_x = ctx->gather(b, 0);
        s.gather_z = ctx->gather(b, 1);
        const size_t eb = strip_elem_bytes(ctx->cfg.strip_precision);
        s.strips = ctx->strips ? static_cast<char*>(ctx->strips) + (size_t)b * ctx->nt * ctx->strip_slot * eb : nullptr;
        s.stage = ctx->stage ? ctx->stage + (size_t)b * 2 * ctx->strip_slot : nullptr;
        s.amax = ctx->amax ? ctx->amax + (size_t)b * ctx->nt * kStripFields : nullptr;
        s.X = w.X;
        s.tiles_x = (w.X + TX - 1) / TX;
        s.rec_tiles_x = rec_tiles_for(w.X, L);
        s.ring = Ring::make(w.X, Z, L, ctx->N);
        s.off = (size_t)b * ctx->shot_stride;
        s.strip_slot = ctx->strip_slot;
        s.vp2 = slot_field(ctx, b, 0); s.vs2 = slot_field(ctx, b, 1);
        s.ax = slot_field(ctx, b, 2); s.az = slot_field(ctx, b, 3);
        s.bx = slot_field(ctx, b, 4); s.bz = slot_field(ctx, b, 5);
    }
    CKS(cudaMemcpyAsync(ctx->d_desc, d.data(), n * sizeof(ShotDesc), cudaMemcpyHostToDevice, ctx->stream));
    return OUC_OK;
}

// Gathers between the caller's layout (X_b x nt or nt x X_b, host) and the
// time-major device gather of width X_b.
int gather_to_device(ouc_ctx* ctx, const float* src, float* dst_tx, int Xb) {
    const size_t n = (size_t)ctx->nt * Xb;
    if (ctx->cfg.gather_layout == OUC_GATHER_TX) {
        CKS(cudaMemcpyAsync(dst_tx, src, n * 4, cudaMemcpyHostToDevice, ctx->stream));
        return OUC_OK;
    }
    CKS(cudaMemcpyAsync(ctx->staging, src, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    launch_transpose(ctx->staging, dst_tx, Xb, ctx->nt, ctx->stream);
    ctx->timing.kernel_launches += 1;
    return OUC_OK;
}

int gather_to_host(ouc_ctx* ctx, const float* src_tx, float* dst, int Xb) {
    const size_t n = (size_t)ctx->nt * Xb;
    const float* from = src_tx;
    if (ctx->cfg.gather_layout == OUC_GATHER_XT) {
        launch_transpose(src_tx, ctx->staging, ctx->nt, Xb, ctx->stream);
        ctx->timing.kernel_launches += 1;
        from = ctx->staging;
    }
    CKS(cudaMemcpyAsync(dst, from, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return OUC_OK;
}

int group(ouc_ctx* ctx, int n, const ouc_shot* shots, const ouc_aperture* ap, const float* d_w, bool forward_only,
          float* const* gx, float* const* gz, const float* const* rx, const float* const* rz, float* const* ipp,
          float* const* ips) {
    std::vector<std::vector<float>> keep;
    int rc = upload_batch(ctx, n, shots, ap, d_w, keep);
    if (rc) return rc;
    const bool self_records = !forward_only && rx == nullptr;
    CKS(cudaEventRecord(ctx->ev[0], ctx->stream));
    if ((rc = run_forward(ctx, n, forward_only || self_records, !forward_only))) return rc;
    if (forward_only) {
        CKS(cudaEventRecord(ctx->ev[1], ctx->stream));
        for (int b = 0; b < n; ++b) {
            const int Xb = ap[b].x1 - ap[b].x0 + 2 * ctx->L;
            if (gx && gx[b] && (rc = gather_to_host(ctx, ctx->gather(b, 0), gx[b], Xb))) return rc;
            if (gz && gz[b] && (rc = gather_to_host(ctx, ctx->gather(b, 1), gz[b], Xb))) return rc;
            // the staging buffer is reused by the next gather
            CKS(cudaStreamSynchronize(ctx->stream));
        }
        ctx->timing.forward_ms += elapsed(ctx->ev[0], ctx->ev[1]);
        return OUC_OK;
    }
    for (int b = 0; b < n && !self_records; ++b) {
        if (!rx[b] || !rz[b]) return fail(ctx, OUC_EINVAL, "record pointer missing for a shot");
        const int Xb = ap[b].x1 - ap[b].x0 + 2 * ctx->L;
        if ((rc = gather_to_device(ctx, rx[b], ctx->gather(b, 0), Xb))) return rc;
        if ((rc = gather_to_device(ctx, rz[b], ctx->gather(b, 1), Xb))) return rc;
        CKS(cudaStreamSynchronize(ctx->stream));   // staging reused
    }
    for (int b = 0; b < n; ++b) {
        if (!shots[b].mute) continue;
        const int L = ctx->L, Xb = ap[b].x1 - ap[b].x0 + 2 * L;
        const int sx = shots[b].sx - ap[b].x0 + L, sz = shots[b].sz + L, rzz = shots[b].rz + L;
        const float v = ctx->vp_host[(size_t)(shots[b].sx + L) * ctx->Z + rzz];   // Vp at (Sx, Z_receive), PS:1645
        launch_mute(ctx->gather(b, 0), ctx->gather(b, 1), Xb, ctx->nt, sx, sz, rzz, shots[b].t0, ctx->cfg.dt,
                    ctx->cfg.dx, v, ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    CKS(cudaEventRecord(ctx->ev[1], ctx->stream));
    const bool theta = shots[0].src_type == OUC_SRC_THETA;
    for (int b = 1; b < n; ++b)
        if ((shots[b].src_type == OUC_SRC_THETA) != theta) return fail(ctx, OUC_EINVAL, "mixed source types in a batch");
    if ((rc = run_backward(ctx, n, ctx->cfg.strip_level == OUC_STRIP_EXACT, theta))) return rc;
    // runtime stability check of the imaging accumulators (as the whole-grid calls do)
    for (int b = 0; b < n; ++b)
        launch_finite_check(ctx->acc[0] - (size_t)kGX * ctx->pitch - kZOFF + (size_t)b * ctx->shot_stride,
                            3 * ctx->fstride, ctx->d_status, ctx->stream);
    CKS(cudaEventRecord(ctx->ev[2], ctx->stream));
    // normalisation + Laplacian per shot, into the stack at the shot's rows
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    for (int b = 0; b < n; ++b) {
        FinalizeArgs f;
        memset(&f, 0, sizeof(f));
        f.X = ap[b].x1 - ap[b].x0 + 2 * ctx->L; f.Z = ctx->Z; f.pitch = ctx->pitch; f.L = ctx->L;
        f.nshots = 1;
        f.shot_stride = ctx->shot_stride;
        f.dh = ctx->cfg.dx;   // main() passes dx as the Laplacian spacing (PS:2372)
        f.illum_scale = 1;
        const size_t off = (size_t)b * ctx->shot_stride;
        for (int k = 0; k < 3; ++k) {
            f.acc[k] = ctx->acc[k] + off;
            f.comp[k] = ctx->cfg.compensated_image ? ctx->comp[k] + off : nullptr;
            f.stack[k] = ctx->d_stack[k] + (size_t)ap[b].x0 * ctx->nz;
        }
        f.img = ctx->d_img + (size_t)(2 * b) * ni;
        f.status = ctx->d_status;
        launch_finalize(f, ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    for (int b = 0; b < n; ++b) {
        const size_t nib = (size_t)(ap[b].x1 - ap[b].x0) * ctx->nz;
        if (ipp && ipp[b]) CKS(cudaMemcpyAsync(ipp[b], ctx->d_img + (size_t)(2 * b) * ni, nib * 4, cudaMemcpyDeviceToHost, ctx->stream));
        if (ips && ips[b]) CKS(cudaMemcpyAsync(ips[b], ctx->d_img + (size_t)(2 * b) * ni + nib, nib * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CKS(cudaEventRecord(ctx->ev[3], ctx->stream));
    CKS(cudaStreamSynchronize(ctx->stream));
    if ((rc = check_status(ctx))) return rc;
    ctx->timing.forward_ms += elapsed(ctx->ev[0], ctx->ev[1]);
    ctx->timing.backward_ms += elapsed(ctx->ev[1], ctx->ev[2]);
    ctx->timing.finalize_ms += elapsed(ctx->ev[2], ctx->ev[3]);
    return OUC_OK;
}

int run(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const ouc_aperture* ap, const float* wavelet,
        bool forward_only, float* const* gx, float* const* gz, const float* const* rx, const float* const* rz,
        float* const* ipp, float* const* ips) {
    if (!ctx) return OUC_EINVAL;
    if (!wavelet) return fail(ctx, OUC_EINVAL, "wavelet is NULL");
    if ((rx == nullptr) != (rz == nullptr)) return fail(ctx, OUC_EINVAL, "give both record components or neither");
    int rc = check(ctx, nshots, shots, ap);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    if (!forward_only && (rc = ensure_strips(ctx))) return rc;
    ctx->timing = ouc_timing{};
    CKS(cudaMemcpyAsync(ctx->d_wavelet, wavelet, (size_t)ctx->nt * 4, cudaMemcpyHostToDevice, ctx->stream));
    for (int s0 = 0; s0 < nshots; s0 += ctx->run_batch) {
        const int n = std::min(ctx->run_batch, nshots - s0);
        auto sub = [&](auto* p) { return p ? p + s0 : nullptr; };
        rc = group(ctx, n, shots + s0, ap + s0, ctx->d_wavelet, forward_only, sub(gx), sub(gz), sub(rx), sub(rz),
                   sub(ipp), sub(ips));
        if (rc) return rc;
    }
    return OUC_OK;
}

// Forward steps per second of n copies of a centre shot (CUDA events).
int time_batch(ouc_ctx* ctx, int n, int steps, float* ms) {
    std::vector<ouc_shot> shots(n);
    for (auto& s : shots) {
        memset(&s, 0, sizeof(s));
        s.sx = ctx->nx / 2; s.sz = std::min(2, ctx->nz - 1); s.rz = s.sz;
    }
    int rc = upload_desc(ctx, n, shots.data(), ctx->d_wavelet);
    if (rc || (rc = zero_side(ctx, n, 0, false))) return rc;
    Side s = ctx->src0;
    StepArgs a = base_args(ctx);
    for (int t = 0; t < 2; ++t)
        if ((rc = fwd_step(ctx, a, s, n, t))) return rc;
    CKS(cudaEventRecord(ctx->ev[0], ctx->stream));
    for (int t = 2; t < 2 + steps; ++t)
        if ((rc = fwd_step(ctx, a, s, n, t % ctx->nt))) return rc;
    CKS(cudaEventRecord(ctx->ev[1], ctx->stream));
    CKS(cudaStreamSynchronize(ctx->stream));
    *ms = elapsed(ctx->ev[0], ctx->ev[1]);
    return OUC_OK;
}

}  // namespace survey
}  // namespace ouc

extern "C" {

int ouc_tune_batch(ouc_ctx* ctx, int steps, int* best_batch, float* ns_per_cell) {
    if (!ctx || steps < 1) return OUC_EINVAL;
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    if (cudaMemsetAsync(ctx->d_wavelet, 0, (size_t)ctx->nt * 4, ctx->stream) != cudaSuccess) return OUC_ECUDA;
    std::vector<int> cands;
    for (int n = 1; n < ctx->batch; n *= 2) cands.push_back(n);
    cands.push_back(ctx->batch);
    int best = 1;
    float best_ns = 0.f;
    for (int n : cands) {
        float ms = 0.f;
        int rc = ouc::survey::time_batch(ctx, n, steps, &ms);
        if (rc) return rc;
        const float ns = ms * 1e6f / ((float)n * steps * ctx->X * ctx->Z);
        // a larger batch must be clearly faster to be preferred (memory per shot)
        if (best_ns == 0.f || ns < 0.97f * best_ns) {
            best = n;
            best_ns = ns;
        }
    }
    ctx->run_batch = best;
    if (best_batch) *best_batch = best;
    if (ns_per_cell) *ns_per_cell = best_ns;
    return OUC_OK;
}

int ouc_tune(ouc_ctx* ctx, int steps, int* best_batch, int* best_seg_rows, float* ns_per_cell) {
    if (!ctx || steps < 1) return OUC_EINVAL;
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    if (cudaMemsetAsync(ctx->d_wavelet, 0, (size_t)ctx->nt * 4, ctx->stream) != cudaSuccess) return OUC_ECUDA;
    std::vector<int> batches, segs = {0, OUC_STEP_TILE_QUEUE};
    for (int n = 1; n < ctx->batch; n *= 2) batches.push_back(n);
    batches.push_back(ctx->batch);
    for (int r : {64, 96, 128, 192, 256, 384, 512})
        if (r < ctx->X + 16) segs.push_back(r);
    int best = 1, best_seg = ctx->seg_rows;
    float best_ns = 0.f;
    for (int n : batches) {
        int seg_n = 0;
        float ns_n = 0.f;
        for (int r : segs) {
            int rc = ouc_set_step_kernel(ctx, r);
            float ms = 0.f;
            if (!rc) rc = ouc::survey::time_batch(ctx, n, steps, &ms);
            if (rc) return rc;
            const float ns = ms * 1e6f / ((float)n * steps * ctx->X * ctx->Z);
            if (ns_n == 0.f || ns < ns_n) { ns_n = ns; seg_n = r; }
        }
        // a larger batch must be clearly faster to be preferred (memory per shot)
        if (best_ns == 0.f || ns_n < 0.97f * best_ns) {
            best = n;
            best_ns = ns_n;
            best_seg = seg_n;
        }
    }
    ctx->run_batch = best;
    const int rc = ouc_set_step_kernel(ctx, best_seg);
    if (rc) return rc;
    if (best_batch) *best_batch = best;
    if (best_seg_rows) *best_seg_rows = best_seg;
    if (ns_per_cell) *ns_per_cell = best_ns;
    return OUC_OK;
}

int ouc_set_run_batch(ouc_ctx* ctx, int n) {
    if (!ctx || n < 1 || n > ctx->batch) return OUC_EINVAL;
    ctx->run_batch = n;
    return OUC_OK;
}

int ouc_survey_forward(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const ouc_aperture* apertures,
                       const float* wavelet, float* const* gather_vx, float* const* gather_vz) {
    return ouc::survey::run(ctx, nshots, shots, apertures, wavelet, true, gather_vx, gather_vz, nullptr, nullptr,
                            nullptr, nullptr);
}

int ouc_survey_rtm(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const ouc_aperture* apertures,
                   const float* wavelet, const float* const* rec_vx, const float* const* rec_vz, float* const* img_pp,
                   float* const* img_ps) {
    return ouc::survey::run(ctx, nshots, shots, apertures, wavelet, false, nullptr, nullptr, rec_vx, rec_vz, img_pp,
                            img_ps);
}

}  // extern "C"
