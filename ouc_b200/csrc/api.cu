// C ABI of libouc.so: context, device memory and the per-shot time loops.
//
// Host-side orchestration that replaces the reference's main() (PS:1658-2401)
// for the modeling and RTM path: model padding and damping profile, the
// forward loop with boundary-strip save, the mute, the backward loop that
// back-propagates the records and reconstructs the source wavefield, the
// imaging condition and the per-shot image finalisation with an FP64 stack.
// Shots of a batch advance together: each time step is one launch per stage
// with blockIdx.y selecting the shot (the reference runs shots one after the
// other, PS:2108).
#include <cuda_runtime.h>

#include <climits>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ouc.h"
#include "ouc_internal.h"
#include "ctx.h"

using namespace ouc;

static_assert((int)OUC_PREC_FP32 == (int)ouc::kStripF32 && (int)OUC_PREC_FP16 == (int)ouc::kStripF16 &&
                  (int)OUC_PREC_BF16 == (int)ouc::kStripBF16,
              "strip precision codes");



namespace ouc {
namespace host {

int fail(ouc_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(ouc_ctx* c, cudaError_t e, const char* what) {
    return fail(c, OUC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);   \
    } while (0)

// Read and clear the context's device status word after a synchronising call:
// a bounded copy wait that gave up, or a non-finite wavefield.
// Tile orders of the dynamic-queue form, heaviest first: tiles whose S
// region meets the damping layers (CPML memories to read and write) and
// tiles that meet the boundary ring (strips to save or restore) lead, then
// the interior tiles; ties in row-major order.  Entries are tx << 16 | tz,
// relative to the launch's tile origin.
std::vector<int> tile_order(const ouc_ctx* ctx, bool rec) {
    const int TX = 32, TZ = 64, SHX = (ctx->N + 1) & ~1, HS = (ctx->N + 3) & ~3;
    const int nx = rec ? ctx->rec_tiles_x : ctx->tiles_x, nz = rec ? ctx->rec_tiles_z : ctx->tiles_z;
    const int ox = rec ? ctx->rec_x0 : 0, oz = rec ? ctx->rec_z0 : 0;
    const int X = ctx->X, Z = ctx->Z, L = ctx->L;
    std::vector<std::pair<int, int>> w;
    for (int tx = 0; tx < nx; ++tx)
        for (int tz = 0; tz < nz; ++tz) {
            const int x0 = ox + tx * TX, z0 = oz + tz * TZ;
            int weight = 0;
            if (!rec && (x0 - SHX < L || x0 + TX + SHX - 1 >= X - L)) weight += 2;
            if (!rec && (z0 - HS < L || z0 + TZ + HS - 1 >= Z - L)) weight += 2;
            const Ring& R = ctx->ring;
            const bool meets_box = x0 - 2 * R.N < X - L + R.N && x0 + TX + 2 * R.N > L - R.N &&
                                   z0 - 2 * R.N < Z - L + R.N && z0 + TZ + 2 * R.N > L - R.N;
            const bool deep = x0 - 2 * R.N >= L + R.N && x0 + TX + 2 * R.N <= X - L - R.N &&
                              z0 - 2 * R.N >= L + R.N && z0 + TZ + 2 * R.N <= Z - L - R.N;
            if (meets_box && !deep) weight += 1;
            w.push_back({-weight, tx * nz + tz});
        }
    std::stable_sort(w.begin(), w.end());
    std::vector<int> out;
    for (auto& e : w) out.push_back(((e.second / nz) << 16) | (e.second % nz));
    return out;
}

int check_status(ouc_ctx* ctx) {
    int st = 0;
    CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (st == 0) return OUC_OK;
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (st & 1) return fail(ctx, OUC_ETIMEOUT, "a step kernel's copy wait timed out");
    return fail(ctx, OUC_EUNSTABLE, "non-finite wavefield (unstable run: check the CFL number and the inputs)");
}


// Edge padding of the interior model into the absorbing layer, as the
// reference's xiangbian (PS:37-119): sides copy the nearest interior
// row/column, corners the nearest interior corner cell.
void pad_edges(std::vector<float>& f, int X, int Z, int L) {
    auto at = [&](int i, int j) -> float& { return f[(size_t)i * Z + j]; };
    for (int i = L; i < X - L; ++i) {
        for (int j = 0; j < L; ++j) at(i, j) = at(i, L);
        for (int j = Z - L; j < Z; ++j) at(i, j) = at(i, Z - L - 1);
    }
    for (int j = L; j < Z - L; ++j) {
        for (int i = 0; i < L; ++i) at(i, j) = at(L, j);
        for (int i = X - L; i < X; ++i) at(i, j) = at(X - L - 1, j);
    }
    for (int i = 0; i < X; ++i) {
        if (i >= L && i < X - L) continue;
        for (int j = 0; j < Z; ++j) {
            if (j >= L && j < Z - L) continue;
            at(i, j) = at(i < L ? L : X - L - 1, j < L ? L : Z - L - 1);
        }
    }
}

// Damping profile of PS:2067-2105: d = log10(1/R) * 1.5 * Vp / L *
// (dist/L)^4 with L in cells, computed in double and stored as float.
// Left/top layers hold L damped cells, right/bottom L-1 (strict ">").
void damping(const std::vector<float>& vp, int X, int Z, int L, double R, std::vector<float>& ax,
             std::vector<float>& az) {
    const double g = log10(1.0 / R) * 1.5;
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Z; ++j) {
            const size_t c = (size_t)i * Z + j;
            const double v = vp[c];
            if (i < L) ax[c] = (float)(g * v / L * pow(1.0 * (L - i) / L, 4.0));
            else if (i > X - L) ax[c] = (float)(g * v / L * pow(1.0 * (i - X + L) / L, 4.0));
            else ax[c] = 0.f;
            if (j < L) az[c] = (float)(g * v / L * pow(1.0 * (L - j) / L, 4.0));
            else if (j > Z - L) az[c] = (float)(g * v / L * pow(1.0 * (j - Z + L) / L, 4.0));
            else az[c] = 0.f;
        }
}

int upload_field(ouc_ctx* ctx, float* dst, const float* host) {
    CK(cudaMemcpy2DAsync(dst, (size_t)ctx->pitch * 4, host, (size_t)ctx->Z * 4, (size_t)ctx->Z * 4, ctx->X,
                         cudaMemcpyHostToDevice, ctx->stream));
    return OUC_OK;
}

StepArgs base_args(const ouc_ctx* c) {
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.X = c->X; a.Z = c->Z; a.pitch = c->pitch; a.L = c->L;
    a.tiles_z = c->tiles_z; a.tile_x0 = 0; a.tile_z0 = 0;
    for (int k = 0; k < 6; ++k) a.a[k] = c->a[k];
    a.dx = c->cfg.dx; a.dz = c->cfg.dz; a.dt = c->cfg.dt;
    a.dt2 = c->cfg.dt * c->cfg.dt;
    a.rdx = 1.0f / c->cfg.dx;   // correctly rounded reciprocal (host IEEE division)
    a.rdz = 1.0f / c->cfg.dz;
    a.vp2 = c->vp2; a.vs2 = c->vs2; a.ax = c->ax; a.az = c->az;
    a.shot_stride = c->shot_stride;
    a.strip_slot = c->strip_slot;
    a.strip_prec = c->cfg.strip_precision;
    a.comp_image = c->cfg.compensated_image;
    a.density = c->cfg.density;
    a.seg_rows = c->seg_rows;
    a.err = c->d_status;
    a.nsm = c->nsm;
    a.queue = c->d_queue;
    a.order[0] = c->d_order[0];
    a.order[1] = c->d_order[1];
    for (int k = 0; k < 3; ++k) a.comp[k] = c->comp[k];
    a.ring = c->ring;
    a.shots = c->d_desc;
    a.box_map = c->box_map;
    a.own_map = c->own_map;
    a.s_map = c->s_map;
    a.state0 = c->box_state0;
    a.fstride = c->fstride;
    a.nfields = kFieldsPerShot;
    a.copy_tx_extra = c->copy_stall ? 16u : 0u;
    return a;
}

void bind_side(StepArgs& a, const Side& s) {
    for (int k = 0; k < 4; ++k) {
        a.now[k] = s.now[k]; a.past[k] = s.past[k];
        a.f_old[k] = s.fo[k]; a.f_new[k] = s.fn[k];
    }
    for (int k = 0; k < 8; ++k) a.o[k] = s.o[k];
}

int check_shot(ouc_ctx* ctx, const ouc_shot* s) {
    if (!s) return fail(ctx, OUC_EINVAL, "shot is NULL");
    if (s->sx < 0 || s->sx >= ctx->nx || s->sz < 0 || s->sz >= ctx->nz)
        return fail(ctx, OUC_EINVAL, "source outside the interior grid");
    if (s->rz < 0 || s->rz >= ctx->nz) return fail(ctx, OUC_EINVAL, "receiver row outside the interior grid");
    if (s->src_type != OUC_SRC_THETA && s->src_type != OUC_SRC_FORCE_Z)
        return fail(ctx, OUC_EINVAL, "unknown source type");
    return OUC_OK;
}

int ensure_strips(ouc_ctx* ctx) {
    if (ctx->strips) return OUC_OK;
    const int prec = ctx->cfg.strip_precision;
    const size_t bytes = ctx->strip_slot * (size_t)ctx->nt * ctx->batch * strip_elem_bytes(prec);
    const size_t stage = prec == kStripF16 ? ctx->strip_slot * 2 * ctx->batch * sizeof(float) : 0;
    const size_t amax = prec == kStripF16 ? (size_t)ctx->nt * kStripFields * ctx->batch * sizeof(unsigned) : 0;
    bool ok = cudaMalloc(&ctx->strips, bytes) == cudaSuccess;
    if (ok && stage) ok = cudaMalloc(&ctx->stage, stage) == cudaSuccess && cudaMalloc(&ctx->amax, amax) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        cudaFree(ctx->strips); cudaFree(ctx->stage); cudaFree(ctx->amax);
        ctx->strips = nullptr; ctx->stage = nullptr; ctx->amax = nullptr;
        return fail(ctx, OUC_ENOMEM, "cannot allocate boundary strips (" + std::to_string((bytes + stage) >> 20) + " MiB)");
    }
    ctx->bytes += bytes + stage + amax;
    return OUC_OK;
}

int ensure_grad(ouc_ctx* ctx) {
    if (ctx->grad) return OUC_OK;
    const size_t bytes = (size_t)ctx->batch * 3 * ctx->fstride * sizeof(float);
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    bool ok = cudaMalloc(&ctx->grad, bytes) == cudaSuccess;
    for (int k = 0; k < 3 && ok; ++k) ok = cudaMalloc(&ctx->d_gstack[k], ni * 8) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return fail(ctx, OUC_ENOMEM, "cannot allocate the gradient accumulators");
    }
    for (int k = 0; k < 3; ++k) CK(cudaMemsetAsync(ctx->d_gstack[k], 0, ni * 8, ctx->stream));
    CK(cudaMemsetAsync(ctx->grad, 0, bytes, ctx->stream));   // guard cells stay zero
    ctx->bytes += bytes + 3 * ni * 8;
    return OUC_OK;
}

int ensure_snaps(ouc_ctx* ctx) {
    if (ctx->snaps) return OUC_OK;
    const int prec = ctx->cfg.strip_precision;
    const size_t elems = (size_t)ctx->nslots * 2 * ctx->nx * ctx->nz * ctx->batch;
    const size_t bytes = elems * strip_elem_bytes(prec);
    const size_t amax = prec == kStripF16 ? (size_t)ctx->nslots * 2 * ctx->batch * sizeof(unsigned) : 0;
    bool ok = cudaMalloc(&ctx->snaps, bytes) == cudaSuccess;
    if (ok && amax) ok = cudaMalloc(&ctx->snap_amax, amax) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        cudaFree(ctx->snaps); cudaFree(ctx->snap_amax);
        ctx->snaps = nullptr; ctx->snap_amax = nullptr;
        return fail(ctx, OUC_ENOMEM, "cannot allocate source snapshots (" + std::to_string(bytes >> 20) + " MiB)");
    }
    ctx->bytes += bytes + amax;
    return OUC_OK;
}

SnapArgs snap_args(const ouc_ctx* ctx, int slot) {
    SnapArgs a;
    memset(&a, 0, sizeof(a));
    a.X = ctx->X; a.Z = ctx->Z; a.pitch = ctx->pitch; a.L = ctx->L; a.nx = ctx->nx; a.nz = ctx->nz;
    a.shot_stride = ctx->shot_stride;
    a.prec = ctx->cfg.strip_precision;
    a.slot = slot;
    a.nslots = ctx->nslots;
    a.shot_elems = (size_t)ctx->nslots * 2 * ctx->nx * ctx->nz;
    a.snaps = ctx->snaps;
    a.amax = ctx->snap_amax;
    a.comp_image = ctx->cfg.compensated_image;
    for (int k = 0; k < 3; ++k) { a.acc[k] = ctx->acc[k]; a.comp[k] = ctx->comp[k]; }
    return a;
}

// Upload the descriptors of n shots (padded coordinates).
int upload_desc(ouc_ctx* ctx, int n, const ouc_shot* shots, const float* d_wavelet) {
    std::vector<ShotDesc> d(n);
    for (int b = 0; b < n; ++b) {
        d[b].sx = shots[b].sx + ctx->L;
        d[b].sz = shots[b].sz + ctx->L;
        d[b].rz = shots[b].rz + ctx->L;
        d[b].src_type = shots[b].src_type;
        d[b].wavelet = d_wavelet;
        d[b].gather_x = ctx->gather(b, 0);
        d[b].gather_z = ctx->gather(b, 1);
        d[b].strips = ctx->strips ? static_cast<char*>(ctx->strips) + (size_t)b * ctx->nt * ctx->strip_slot *
                                                                   strip_elem_bytes(ctx->cfg.strip_precision)
                                  : nullptr;
        d[b].stage = ctx->stage ? ctx->stage + (size_t)b * 2 * ctx->strip_slot : nullptr;
        d[b].amax = ctx->amax ? ctx->amax + (size_t)b * ctx->nt * kStripFields : nullptr;
        d[b].X = ctx->X;
        d[b].tiles_x = ctx->tiles_x;
        d[b].rec_tiles_x = ctx->rec_tiles_x;
        d[b].ring = ctx->ring;
        d[b].off = (size_t)b * ctx->shot_stride;
        d[b].strip_slot = ctx->strip_slot;
        d[b].vp2 = ctx->vp2; d[b].vs2 = ctx->vs2; d[b].ax = ctx->ax; d[b].az = ctx->az;
        d[b].bx = ctx->bx; d[b].bz = ctx->bz;
    }
    CK(cudaMemcpyAsync(ctx->d_desc, d.data(), n * sizeof(ShotDesc), cudaMemcpyHostToDevice, ctx->stream));
    return OUC_OK;
}

// Zero the source- or receiver-side fields (and optionally the accumulators)
// of n shots.
int zero_side(ouc_ctx* ctx, int n, int side, bool with_acc) {
    for (int b = 0; b < n; ++b) {
        float* base = ctx->state + (size_t)b * ctx->shot_stride + (size_t)side * kFieldsPerSide * ctx->fstride;
        CK(cudaMemsetAsync(base, 0, (size_t)kFieldsPerSide * ctx->fstride * sizeof(float), ctx->stream));
        if (with_acc) {
            float* acc = ctx->state + (size_t)b * ctx->shot_stride + (size_t)2 * kFieldsPerSide * ctx->fstride;
            CK(cudaMemsetAsync(acc, 0, (size_t)6 * ctx->fstride * sizeof(float), ctx->stream));   // acc + comp
        }
    }
    return OUC_OK;
}

// One forward step of n shots at time t (forward_s + forward_u with the
// receiver record and the strip save, PS:2261-2266); `a` carries record/save.
int fwd_step(ouc_ctx* ctx, StepArgs& a, Side& s, int n, int t) {
    bind_side(a, s);
    a.t = t;
    if (launch_step(ctx->N, kFwd, a, ctx->tiles_x, n, ctx->stream))
        return fail(ctx, OUC_EINVAL, "step launch refused (half-order or state map)");
    s.swap_levels();
    s.swap_memory();
    ctx->timing.kernel_launches += 1;
    return OUC_OK;
}

// Run `body` (a whole-shot time loop that enqueues work on the context
// stream and may set ctx->src) directly, or, with cfg.use_graphs, as a CUDA
// graph: captured on first use for its key and replayed afterwards.  Every
// launch argument of a loop depends only on the key and on fixed context
// buffers (per-batch values travel in the shot descriptors), so one graph
// serves every batch with that key.
template <class F>
int with_graph(ouc_ctx* ctx, const int (&key)[6], F&& body) {
    if (!ctx->cfg.use_graphs) return body();
    for (const auto& g : ctx->graphs) {
        if (std::equal(key, key + 6, g.key)) {
            CK(cudaGraphLaunch(g.exec, ctx->stream));
            ctx->src = g.src_end;
            ctx->timing.kernel_launches += g.launches;
            return OUC_OK;
        }
    }
    const long long before = ctx->timing.kernel_launches;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return rc ? rc : cuda_fail(ctx, e, "graph capture");
    }
    ouc_ctx::Graph g;
    std::copy(key, key + 6, g.key);
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return cuda_fail(ctx, ei, "graph instantiation");
    g.src_end = ctx->src;
    g.launches = ctx->timing.kernel_launches - before;
    ctx->graphs.push_back(g);
    CK(cudaGraphLaunch(g.exec, ctx->stream));
    return OUC_OK;
}

// Forward time loop (PS:2258-2292) of n shots.  Records into the time-major
// gathers when `record`, saves the boundary ring of every step when `save`.
int run_forward(ouc_ctx* ctx, int n, bool record, bool save, bool snaps) {
    const int key[6] = {0, n, record, save, snaps, 0};
    return with_graph(ctx, key, [&]() { return run_forward_loop(ctx, n, record, save, snaps); });
}

int run_forward_loop(ouc_ctx* ctx, int n, bool record, bool save, bool snaps) {
    Side s = ctx->src0;   // state zeroed below: start from the fixed buffer assignment
    int rc = zero_side(ctx, n, 0, false);
    if (rc) return rc;
    StepArgs a = base_args(ctx);
    a.record = record;
    a.save = save;
    const bool f16 = save && ctx->cfg.strip_precision == kStripF16;
    if (f16) CK(cudaMemsetAsync(ctx->amax, 0, (size_t)n * ctx->nt * kStripFields * sizeof(unsigned), ctx->stream));
    if (snaps && ctx->snap_amax)
        CK(cudaMemsetAsync(ctx->snap_amax, 0, (size_t)n * ctx->nslots * 2 * sizeof(unsigned), ctx->stream));
    for (int t = 0; t < ctx->nt; ++t) {
        if ((rc = fwd_step(ctx, a, s, n, t))) return rc;
        if (snaps && ctx->snap_fwd[t] >= 0) {   // the new level is an imaging level: keep it
            SnapArgs sa = snap_args(ctx, ctx->snap_fwd[t]);
            sa.px = s.now[0];
            sa.pz = s.now[1];
            launch_snap_store(sa, n, ctx->stream);
            ctx->timing.kernel_launches += ctx->snap_amax ? 2 : 1;
        }
    }
    if (f16) {   // the last slot: its maxima are complete now
        launch_strip_pack(ctx->d_desc, n, ctx->nt - 1, ctx->ring.R, ctx->strip_slot, ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    ctx->src = s;
    CK(cudaGetLastError());
    return OUC_OK;
}

// Launch arguments of the two backward wavefields.
StepArgs rcv_args(const ouc_ctx* ctx) { return base_args(ctx); }

StepArgs rec_args(const ouc_ctx* ctx) {
    StepArgs as = base_args(ctx);
    as.tiles_z = ctx->rec_tiles_z; as.tile_x0 = ctx->rec_x0; as.tile_z0 = ctx->rec_z0;
    as.img_past = ctx->cfg.image_align == OUC_IMAGE_REFERENCE;
    for (int k = 0; k < 3; ++k) as.acc[k] = ctx->acc[k];
    return as;
}

// Receiver side at time t: record injection + S/U stages with damping
// (PS:2319-2324, 2349-2354).
int rcv_step(ouc_ctx* ctx, StepArgs& ar, Side& r, int n, int t, cudaStream_t st = nullptr) {
    bind_side(ar, r);
    ar.t = t;
    if (launch_step(ctx->N, kRcv, ar, ctx->tiles_x, n, st ? st : ctx->stream))
        return fail(ctx, OUC_EINVAL, "step launch refused (half-order or state map)");
    r.swap_levels();
    r.swap_memory();
    ctx->timing.kernel_launches += 1;
    return OUC_OK;
}

// Source side at time t, after rcv_step(t): inverse leapfrog on the interior
// from levels t+1 and t+2 with the strip restore, and the imaging condition
// (PS:2326-2361).  At t = nt-1 there is no reconstruction: the forward's
// final level is correlated as it stands.
int rec_step(ouc_ctx* ctx, StepArgs& as, Side& s, const Side& r, int n, int t, bool exact_strips, bool theta_src) {
    const int nt = ctx->nt;
    if (t == nt - 1) {
        StepArgs ai = base_args(ctx);
        for (int k = 0; k < 4; ++k) { ai.now[k] = s.now[k]; ai.rcv[k] = r.now[k]; }
        for (int k = 0; k < 3; ++k) ai.acc[k] = ctx->acc[k];
        launch_image_only(ai, n, ctx->stream);
        ctx->timing.kernel_launches += 1;
        s.swap_levels();   // now = level NT-1, past = level NT
        return OUC_OK;
    }
    bind_side(as, s);
    as.t = t;
    as.src_recon = theta_src && (exact_strips || t + 1 == nt - 1);
    as.slot_u = exact_strips ? t : (t + 1 == nt - 1 ? nt - 2 : t + 1);
    as.slot_s = t + 1;
    for (int k = 0; k < 4; ++k) as.rcv[k] = r.now[k];
    if (launch_step(ctx->N, kRec, as, ctx->rec_tiles_x, n, ctx->stream))
        return fail(ctx, OUC_EINVAL, "step launch refused (half-order or state map)");
    s.swap_levels();
    ctx->timing.kernel_launches += 1;
    return OUC_OK;
}

// Backward loop (PS:2313-2364) and imaging of n shots; the source side
// holds the forward's last two levels on entry.
// FWI gradient of back-step t, launched between the receiver step and the
// reconstruction: the source level the imaging condition correlates at this
// step (the forward's last level at t = nt-1), the receiver after the step.
void grad_step(ouc_ctx* ctx, const Side& s, const Side& r, int n, int t) {
    GradArgs g;
    memset(&g, 0, sizeof(g));
    g.X = ctx->X; g.Z = ctx->Z; g.pitch = ctx->pitch; g.L = ctx->L; g.N = ctx->N;
    g.nshots = n;
    for (int k = 0; k < 6; ++k) g.a[k] = ctx->a[k];
    g.dx = ctx->cfg.dx; g.dz = ctx->cfg.dz;
    const bool past = t < ctx->nt - 1 && ctx->cfg.image_align == OUC_IMAGE_REFERENCE;
    for (int k = 0; k < 4; ++k) { g.src[k] = past ? s.past[k] : s.now[k]; g.rcv[k] = r.now[k]; }
    g.shot_stride = ctx->shot_stride;
    g.vp = ctx->vpv; g.vs = ctx->vsv; g.rho = ctx->rhov;
    for (int k = 0; k < 3; ++k) g.g[k] = ctx->grad + (size_t)k * ctx->fstride + (size_t)kGX * ctx->pitch + kZOFF;
    g.grad_stride = 3 * ctx->fstride;
    launch_grad(g, ctx->stream);
    ctx->timing.kernel_launches += 1;
}

int run_backward(ouc_ctx* ctx, int n, bool exact_strips, bool theta_src) {
    const int key[6] = {1, n, exact_strips, theta_src, 0, ctx->cfg.gradient};
    return with_graph(ctx, key, [&]() { return run_backward_loop(ctx, n, exact_strips, theta_src); });
}

int run_backward_loop(ouc_ctx* ctx, int n, bool exact_strips, bool theta_src) {
    Side s = ctx->src;    // the forward's last two levels
    Side r = ctx->rcv0;
    int rc = zero_side(ctx, n, 1, true);
    if (rc) return rc;
    if (ctx->cfg.gradient) CK(cudaMemsetAsync(ctx->grad, 0, (size_t)n * 3 * ctx->fstride * sizeof(float), ctx->stream));
    StepArgs ar = rcv_args(ctx);
    StepArgs as = rec_args(ctx);
    if (ctx->cfg.gradient || !ctx->stream2) {
        for (int t = ctx->nt - 1; t >= 0; --t) {
            if ((rc = rcv_step(ctx, ar, r, n, t))) return rc;
            if (ctx->cfg.gradient) grad_step(ctx, s, r, n, t);
            if ((rc = rec_step(ctx, as, s, r, n, t, exact_strips, theta_src))) return rc;
        }
        CK(cudaGetLastError());
        return OUC_OK;
    }
    // Two streams, so that the reconstruction of step t overlaps the
    // receiver step t-1: rec(t) reads the receiver level rcv(t) wrote and
    // rcv(t-1) only reads it too (it writes the older buffer), so the two are
    // independent; rcv(t-2) overwrites that level and waits for rec(t).  The
    // source side stays in order on the context stream.  Same launches, same
    // arguments, same results as the serial loop.
    cudaStream_t sr = ctx->stream2;
    CK(cudaEventRecord(ctx->evb[0], ctx->stream));   // the receiver stream starts after the work queued so far
    CK(cudaStreamWaitEvent(sr, ctx->evb[0], 0));
    for (int t = ctx->nt - 1; t >= 0; --t) {
        if (t <= ctx->nt - 3) CK(cudaStreamWaitEvent(sr, ctx->evb[1 + (t & 1)], 0));   // rec(t+2) is done
        if ((rc = rcv_step(ctx, ar, r, n, t, sr))) return rc;
        CK(cudaEventRecord(ctx->evb[0], sr));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->evb[0], 0));                          // rcv(t) is done
        if ((rc = rec_step(ctx, as, s, r, n, t, exact_strips, theta_src))) return rc;
        CK(cudaEventRecord(ctx->evb[1 + (t & 1)], ctx->stream));
    }
    // rec(0) waited for rcv(0), the receiver stream's last work: joined
    CK(cudaGetLastError());
    return OUC_OK;
}

// Backward loop of the snapshot form: receiver back-propagation at every
// step, imaging at the snapshot levels only.
int run_backward_snap(ouc_ctx* ctx, int n) {
    const int key[6] = {2, n, 0, 0, 0, 0};
    return with_graph(ctx, key, [&]() { return run_backward_snap_loop(ctx, n); });
}

int run_backward_snap_loop(ouc_ctx* ctx, int n) {
    Side r = ctx->rcv0;
    int rc = zero_side(ctx, n, 1, true);
    if (rc) return rc;
    StepArgs ar = rcv_args(ctx);
    for (int t = ctx->nt - 1; t >= 0; --t) {
        if ((rc = rcv_step(ctx, ar, r, n, t))) return rc;
        if (ctx->snap_bwd[t] >= 0) {
            SnapArgs sa = snap_args(ctx, ctx->snap_bwd[t]);
            for (int k = 0; k < 4; ++k) sa.rcv[k] = r.now[k];
            launch_image_snap(sa, n, ctx->stream);
            ctx->timing.kernel_launches += 1;
        }
    }
    CK(cudaGetLastError());
    return OUC_OK;
}

int finalize(ouc_ctx* ctx, int n) {
    FinalizeArgs f;
    f.X = ctx->X; f.Z = ctx->Z; f.pitch = ctx->pitch; f.L = ctx->L;
    f.nshots = n;
    f.shot_stride = ctx->shot_stride;
    f.dh = ctx->cfg.dx;   // main() passes dx as the Laplacian spacing (PS:2372)
    f.illum_scale = ctx->cfg.snapshot_every > 0 ? ctx->cfg.snapshot_every : 1;
    for (int k = 0; k < 3; ++k) {
        f.acc[k] = ctx->acc[k];
        f.comp[k] = ctx->cfg.compensated_image ? ctx->comp[k] : nullptr;
        f.stack[k] = ctx->d_stack[k];
    }
    f.img = ctx->d_img;
    f.status = ctx->d_status;
    launch_finalize(f, ctx->stream);
    ctx->timing.kernel_launches += 1;
    CK(cudaGetLastError());
    return OUC_OK;
}

// Bring a gather from the caller's layout into the time-major device gather.
int gather_in(ouc_ctx* ctx, const float* src, float* dst_tx, bool host) {
    const size_t n = (size_t)ctx->nt * ctx->X;
    const bool xt = ctx->cfg.gather_layout == OUC_GATHER_XT;
    if (!xt) {
        CK(cudaMemcpyAsync(dst_tx, src, n * 4, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream));
        return OUC_OK;
    }
    const float* from = src;
    if (host) {
        CK(cudaMemcpyAsync(ctx->staging, src, n * 4, cudaMemcpyHostToDevice, ctx->stream));
        from = ctx->staging;
    }
    launch_transpose(from, dst_tx, ctx->X, ctx->nt, ctx->stream);   // [X][nt] -> [nt][X]
    ctx->timing.kernel_launches += 1;
    return OUC_OK;
}

int gather_out(ouc_ctx* ctx, const float* src_tx, float* dst, bool host) {
    const size_t n = (size_t)ctx->nt * ctx->X;
    const bool xt = ctx->cfg.gather_layout == OUC_GATHER_XT;
    const float* from = src_tx;
    if (xt) {
        float* tgt = host ? ctx->staging : dst;
        launch_transpose(src_tx, tgt, ctx->nt, ctx->X, ctx->stream);   // [nt][X] -> [X][nt]
        ctx->timing.kernel_launches += 1;
        from = tgt;
        if (!host) return OUC_OK;
    }
    CK(cudaMemcpyAsync(dst, from, n * 4, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
    return OUC_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace host
}  // namespace ouc

using namespace ouc::host;

extern "C" {

const char* ouc_strerror(int status) {
    switch (status) {
        case OUC_OK: return "ok";
        case OUC_EINVAL: return "invalid argument";
        case OUC_ECUDA: return "CUDA runtime error";
        case OUC_ENOMEM: return "device out of memory";
        case OUC_EUNSTABLE: return "unstable configuration (CFL) or non-finite wavefield";
        case OUC_ESTATE: return "call out of order";
        case OUC_ETIMEOUT: return "device wait timed out";
        case OUC_ENODEV: return "no usable sm_100 device";
        case OUC_ESCRATCH: return "problem larger than the fixed scratch of the no-allocation entry point";
    }
    return "unknown status";
}

const char* ouc_last_error(const ouc_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }



int ouc_version(void) { return OUC_VERSION_MAJOR * 100 + OUC_VERSION_MINOR; }

int ouc_stencil_weights(int half_order, float* out) {
    if (half_order < 1 || half_order > 6 || !out) return OUC_EINVAL;
    for (int k = 0; k < half_order; ++k) out[k] = (float)kStencilWeights[half_order][k];
    return OUC_OK;
}

int ouc_ricker(float fm, float dt, int nt, float* out, int* t0_out) {
    if (!(fm > 0) || !(dt > 0) || nt < 1 || !out) return OUC_EINVAL;
    const double pi_ref = 3.1415926;   // PS:14
    const double f = fm;
    const float nk = (float)(pi_ref * pi_ref * f * f * dt * dt);
    const int t0 = (int)ceil(1.0 / (f * dt));
    for (int t = 0; t < nt; ++t) {
        const int d = t - t0;
        const float e = std::exp(-nk * d * d);   // float exponent, as in PS:1958
        out[t] = (float)((1.0 - 2.0 * nk * d * d) * e);
    }
    if (t0_out) *t0_out = t0;
    return OUC_OK;
}

int ouc_create(const ouc_config* cfg, const float* vp, const float* vs, const float* rho, ouc_ctx** out) {
    (void)rho;   // density does not enter the reference's equations (PS:373-378)
    if (!cfg || !vp || !vs || !out) return OUC_EINVAL;
    *out = nullptr;
    ouc_ctx* ctx = new (std::nothrow) ouc_ctx();
    if (!ctx) return OUC_ENOMEM;
    ctx->cfg = *cfg;
    const int N = cfg->half_order, L = cfg->npml;
    auto bad = [&](const std::string& m, int code = OUC_EINVAL) {
        ctx->err = m;
        ouc_destroy(ctx);
        return code;
    };
    if (N != 2 && N != 5 && N != 6) return bad("half_order must be 2, 5 or 6");
    if (cfg->nx < 4 * N || cfg->nz < 4 * N) return bad("interior must be at least 4N cells in each direction");
    if (L < N) return bad("npml must be at least the stencil half-width");
    if (!(cfg->dx > 0) || !(cfg->dz > 0) || !(cfg->dt > 0) || cfg->nt < 2) return bad("bad spacing, time step or nt");
    // the corrected-reciprocal division is exact for quotients above 2^-120,
    // which the 2^-112 accumulator guard ensures for spacings up to 256
    if (cfg->dx > 256.f || cfg->dz > 256.f) return bad("grid spacing above 256 is not supported");
    if (!(cfg->pml_r > 0 && cfg->pml_r < 1)) return bad("pml_r must be in (0, 1)");
    if (cfg->max_batch < 0 || cfg->max_batch > 256) return bad("max_batch must be in [0, 256]");
    {   // one field (guard rows and columns, padded to whole tiles) must stay
        // below 2^31 cells: the kernels address within a field with 32-bit offsets
        const long long Xp = (long long)cfg->nx + 2LL * L, Zp = (long long)cfg->nz + 2LL * L;
        // (bounds of TileGrid's Xc, Zc: one more tile row and column)
        const long long rows = (Xp + 31) / 32 * 32 + 32 + 2LL * kGX;
        const long long pitch = ((Zp + 63) / 64 * 64 + 64 + 2LL * kZOFF + 31) / 32 * 32;
        if (rows * pitch > (long long)INT_MAX) return bad("grid too large: one field would exceed 2^31 cells");
    }
    if (cfg->strip_precision != OUC_PREC_FP32 && cfg->strip_precision != OUC_PREC_FP16 &&
        cfg->strip_precision != OUC_PREC_BF16)
        return bad("strip_precision must be OUC_PREC_FP32, OUC_PREC_FP16 or OUC_PREC_BF16");
    if (cfg->compensated_image != 0 && cfg->compensated_image != 1) return bad("compensated_image must be 0 or 1");
    if (cfg->density != 0 && cfg->density != 1) return bad("density must be 0 or 1");
    if (cfg->gradient != 0 && cfg->gradient != 1) return bad("gradient must be 0 or 1");
    if (cfg->gradient && (cfg->density || cfg->snapshot_every > 0))
        return bad("the FWI gradient runs with the density-normalised equations and the strip form");
    if (cfg->snapshot_every < 0 || cfg->snapshot_every > cfg->nt) return bad("snapshot_every must be in [0, nt]");
    ctx->N = N; ctx->L = L; ctx->nx = cfg->nx; ctx->nz = cfg->nz; ctx->nt = cfg->nt;
    ctx->X = cfg->nx + 2 * L; ctx->Z = cfg->nz + 2 * L;
    ctx->batch = std::max(1, cfg->max_batch);
    ctx->run_batch = ctx->batch;
    for (int k = 0; k < N; ++k) ctx->a[k] = (float)kStencilWeights[N][k];
    const int X = ctx->X, Z = ctx->Z;

    // model on the padded grid
    std::vector<float> P_vp((size_t)X * Z), P_vs((size_t)X * Z);
    if (cfg->model_layout == OUC_MODEL_PADDED) {
        std::copy(vp, vp + (size_t)X * Z, P_vp.begin());
        std::copy(vs, vs + (size_t)X * Z, P_vs.begin());
    } else {
        for (int i = 0; i < cfg->nx; ++i)
            for (int j = 0; j < cfg->nz; ++j) {
                P_vp[(size_t)(i + L) * Z + j + L] = vp[(size_t)i * cfg->nz + j];
                P_vs[(size_t)(i + L) * Z + j + L] = vs[(size_t)i * cfg->nz + j];
            }
        pad_edges(P_vp, X, Z, L);
        pad_edges(P_vs, X, Z, L);
    }
    float vmax = 0.f;
    for (float v : P_vp) {
        if (!(v > 0) || !std::isfinite(v)) return bad("Vp must be positive and finite");
        vmax = std::max(vmax, v);
    }
    for (float v : P_vs)
        if (!(v >= 0) || !std::isfinite(v)) return bad("Vs must be non-negative and finite");
    // stability of the staggered leapfrog: dt vmax sum|a_k| sqrt(1/dx^2 + 1/dz^2) <= 1
    double sa = 0;
    for (int k = 0; k < N; ++k) sa += fabs(kStencilWeights[N][k]);
    const double cfl = cfg->dt * vmax * sa * sqrt(1.0 / (cfg->dx * cfg->dx) + 1.0 / (cfg->dz * cfg->dz));
    if (cfl > 1.0) return bad("CFL number " + std::to_string(cfl) + " > 1 for this dt", OUC_EUNSTABLE);
    std::vector<float> hax((size_t)X * Z), haz((size_t)X * Z);
    damping(P_vp, X, Z, L, cfg->pml_r, hax, haz);
    ctx->vp_host = P_vp;
    std::vector<float> vp2((size_t)X * Z), vs2((size_t)X * Z);
    for (size_t k = 0; k < vp2.size(); ++k) { vp2[k] = P_vp[k] * P_vp[k]; vs2[k] = P_vs[k] * P_vs[k]; }
    // variable density (no counterpart in the reference, whose equations are
    // density-normalised, PS:373-378): moduli rho Vp^2, rho Vs^2 at the cells,
    // buoyancy averaged onto the staggered Ux (i + 1/2) and Uz (j + 1/2) positions
    std::vector<float> hbx, hbz, P_rho;
    if (cfg->density && !rho) return bad("density = 1 needs a density model");
    if (rho) {   // padded density: the variable-density equations and the FWI gradient formula
        P_rho.resize((size_t)X * Z);
        if (cfg->model_layout == OUC_MODEL_PADDED) {
            std::copy(rho, rho + (size_t)X * Z, P_rho.begin());
        } else {
            for (int i = 0; i < cfg->nx; ++i)
                for (int j = 0; j < cfg->nz; ++j) P_rho[(size_t)(i + L) * Z + j + L] = rho[(size_t)i * cfg->nz + j];
            pad_edges(P_rho, X, Z, L);
        }
        for (float v : P_rho)
            if (!(v > 0) || !std::isfinite(v)) return bad("density must be positive and finite");
    }
    if (cfg->density) {
        hbx.resize((size_t)X * Z);
        hbz.resize((size_t)X * Z);
        for (int i = 0; i < X; ++i)
            for (int j = 0; j < Z; ++j) {
                const size_t k = (size_t)i * Z + j;
                vp2[k] = vp2[k] * P_rho[k];
                vs2[k] = vs2[k] * P_rho[k];
                const double b = 1.0 / P_rho[k];
                const double bxn = i + 1 < X ? 1.0 / P_rho[k + Z] : b, bzn = j + 1 < Z ? 1.0 / P_rho[k + 1] : b;
                hbx[k] = (float)(0.5 * (b + bxn));
                hbz[k] = (float)(0.5 * (b + bzn));
            }
    }

    // device
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0) {
        cudaGetLastError();
        return bad("no CUDA device", OUC_ENODEV);
    }
    ctx->device = cfg->device;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return bad("cudaSetDevice failed", OUC_ENODEV);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, ctx->device);
    if (prop.major != 10) return bad(std::string("device ") + prop.name + " is not sm_100", OUC_ENODEV);
    if (cfg->stream) {
        ctx->stream = (cudaStream_t)cfg->stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bad("cannot create stream", OUC_ECUDA);
        ctx->own_stream = true;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    // second stream and ordering events of the overlapped backward loop
    if (cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking) != cudaSuccess) return bad("cannot create stream", OUC_ECUDA);
    for (auto& e : ctx->evb)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return bad("cannot create events", OUC_ECUDA);

    // layout
    const TileGrid tg = tile_grid(X, Z, L);
    ctx->tiles_x = tg.tiles_x; ctx->tiles_z = tg.tiles_z;
    ctx->Xc = tg.Xc; ctx->Zc = tg.Zc;
    ctx->pitch = ((kZOFF + ctx->Zc + kZOFF) + 31) / 32 * 32;
    ctx->fstride = (size_t)(ctx->Xc + 2 * kGX) * ctx->pitch;   // < 2^31 (checked above)
    ctx->shot_stride = (size_t)kFieldsPerShot * ctx->fstride;
    ctx->rec_x0 = tg.rec_x0; ctx->rec_z0 = tg.rec_z0;
    ctx->rec_tiles_x = tg.rec_tiles_x; ctx->rec_tiles_z = tg.rec_tiles_z;
    ctx->ring = Ring::make(X, Z, L, N);
    ctx->strip_slot = (size_t)kStripFields * ctx->ring.R;
    if (cfg->snapshot_every > 0) {
        // imaging steps t = nt-1, nt-1-K, ...; step t correlates the source
        // level t+1 (EXACT, and the last step) or t+2 (REFERENCE, PS:2361),
        // i.e. the new level of forward step t or t+1: one slot per distinct
        // forward step
        const int K = cfg->snapshot_every, nt = cfg->nt;
        ctx->snap_fwd.assign(nt, -1);
        ctx->snap_bwd.assign(nt, -1);
        for (int t = nt - 1; t >= 0; t -= K) {
            const int f = (cfg->image_align == OUC_IMAGE_EXACT || t == nt - 1) ? t : t + 1;
            if (ctx->snap_fwd[f] < 0) ctx->snap_fwd[f] = ctx->nslots++;
            ctx->snap_bwd[t] = ctx->snap_fwd[f];
        }
    }

    const size_t model_bytes = 9 * ctx->fstride * sizeof(float);
    const size_t state_bytes = ctx->shot_stride * ctx->batch * sizeof(float);
    const size_t ng = (size_t)ctx->nt * X;
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    const size_t stage = std::max(ng, (size_t)4 * X * Z);
    bool ok = cudaMalloc(&ctx->model, model_bytes) == cudaSuccess &&
              cudaMalloc(&ctx->state, state_bytes) == cudaSuccess &&
              cudaMalloc(&ctx->gathers, 2 * ng * ctx->batch * 4) == cudaSuccess &&
              cudaMalloc(&ctx->staging, stage * 4) == cudaSuccess &&
              cudaMalloc(&ctx->d_wavelet, (size_t)ctx->nt * 4) == cudaSuccess &&
              cudaMalloc(&ctx->d_img, 2 * ni * ctx->batch * 4) == cudaSuccess &&
              cudaMalloc(&ctx->d_desc, ctx->batch * sizeof(ShotDesc)) == cudaSuccess &&
              cudaMalloc(&ctx->d_status, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&ctx->d_queue, 6 * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&ctx->d_order[0], (size_t)ctx->tiles_x * ctx->tiles_z * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&ctx->d_order[1], (size_t)ctx->rec_tiles_x * ctx->rec_tiles_z * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&ctx->d_stack[0], ni * 8) == cudaSuccess && cudaMalloc(&ctx->d_stack[1], ni * 8) == cudaSuccess &&
              cudaMalloc(&ctx->d_stack[2], ni * 8) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return bad("cannot allocate wavefield state, gathers, images or stack", OUC_ENOMEM);
    }
    ctx->bytes += model_bytes + state_bytes + 2 * ng * ctx->batch * 4 + stage * 4 + (size_t)ctx->nt * 4 +
                  2 * ni * ctx->batch * 4 + 3 * ni * 8;
    // guards and padding of every field must stay zero: clear everything once
    cudaMemsetAsync(ctx->model, 0, model_bytes, ctx->stream);
    cudaMemsetAsync(ctx->state, 0, state_bytes, ctx->stream);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
    cudaMemsetAsync(ctx->d_queue, 0, 6 * sizeof(int), ctx->stream);
    {
        const std::vector<int> o0 = tile_order(ctx, false), o1 = tile_order(ctx, true);
        cudaMemcpyAsync(ctx->d_order[0], o0.data(), o0.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(ctx->d_order[1], o1.data(), o1.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
        cudaStreamSynchronize(ctx->stream);   // the host vectors go out of scope
    }
    cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    ctx->seg_rows = 0;   // the tile kernel; ouc_tune / ouc_set_step_kernel choose the march
    for (int q = 0; q < 3; ++q) cudaMemsetAsync(ctx->d_stack[q], 0, ni * 8, ctx->stream);
    ctx->vp2 = ctx->field(ctx->model, 0); ctx->vs2 = ctx->field(ctx->model, 1);
    ctx->ax = ctx->field(ctx->model, 2); ctx->az = ctx->field(ctx->model, 3);
    ctx->bx = ctx->field(ctx->model, 4); ctx->bz = ctx->field(ctx->model, 5);
    ctx->vpv = ctx->field(ctx->model, 6); ctx->vsv = ctx->field(ctx->model, 7);
    ctx->rhov = P_rho.empty() ? nullptr : ctx->field(ctx->model, 8);
    size_t k = 0;
    for (Side* s : {&ctx->src, &ctx->rcv}) {
        for (int q = 0; q < 4; ++q) s->now[q] = ctx->field(ctx->state, k++);
        for (int q = 0; q < 4; ++q) s->past[q] = ctx->field(ctx->state, k++);
        for (int q = 0; q < 4; ++q) s->fo[q] = ctx->field(ctx->state, k++);
        for (int q = 0; q < 4; ++q) s->fn[q] = ctx->field(ctx->state, k++);
        for (int q = 0; q < 8; ++q) s->o[q] = ctx->field(ctx->state, k++);
    }
    for (int q = 0; q < 3; ++q) ctx->acc[q] = ctx->field(ctx->state, k++);
    for (int q = 0; q < 3; ++q) ctx->comp[q] = ctx->field(ctx->state, k++);
    ctx->src0 = ctx->src;
    ctx->rcv0 = ctx->rcv;
    {   // the state block's tensor map (U boxes of the step kernels)
        StepArgs m;
        memset(&m, 0, sizeof(m));
        if (encode_box_map(m, ctx->state, ctx->pitch, ctx->Xc + 2 * kGX, kFieldsPerShot, ctx->batch, ctx->fstride, N) !=
            cudaSuccess)
            return bad("cannot encode the state block's tensor map", OUC_ECUDA);
        ctx->box_map = m.box_map;
        ctx->own_map = m.own_map;
        ctx->s_map = m.s_map;
        ctx->box_state0 = m.state0;
    }
    // kernel attributes set before any graph capture
    if (configure_step_kernels(N) != cudaSuccess) {
        cudaGetLastError();
        return bad("cannot set the step kernels' shared-memory attributes", OUC_ECUDA);
    }
    int rc = OUC_OK;
    if ((rc = upload_field(ctx, ctx->vp2, vp2.data())) || (rc = upload_field(ctx, ctx->vs2, vs2.data())) ||
        (rc = upload_field(ctx, ctx->ax, hax.data())) || (rc = upload_field(ctx, ctx->az, haz.data())) ||
        (cfg->density && ((rc = upload_field(ctx, ctx->bx, hbx.data())) || (rc = upload_field(ctx, ctx->bz, hbz.data())))) ||
        (rc = upload_field(ctx, ctx->vpv, P_vp.data())) || (rc = upload_field(ctx, ctx->vsv, P_vs.data())) ||
        (ctx->rhov && (rc = upload_field(ctx, ctx->rhov, P_rho.data())))) {
        ouc_destroy(ctx);
        return rc;
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return bad("setup failed", OUC_ECUDA);
    *out = ctx;
    return OUC_OK;
}

int ouc_destroy(ouc_ctx* ctx) {
    if (!ctx) return OUC_OK;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->model); cudaFree(ctx->state);
    cudaFree(ctx->gathers); cudaFree(ctx->staging); cudaFree(ctx->d_wavelet);
    cudaFree(ctx->d_img); cudaFree(ctx->d_desc); cudaFree(ctx->d_status);
    cudaFree(ctx->d_queue); cudaFree(ctx->d_order[0]); cudaFree(ctx->d_order[1]);
    for (auto* p : ctx->d_stack) cudaFree(p);
    cudaFree(ctx->strips); cudaFree(ctx->stage); cudaFree(ctx->amax);
    cudaFree(ctx->snaps); cudaFree(ctx->snap_amax);
    cudaFree(ctx->l_in); cudaFree(ctx->l_out); cudaFree(ctx->l_truth); cudaFree(ctx->l_scale); cudaFree(ctx->l_tmp); cudaFree(ctx->sv_model);
    cudaFree(ctx->grad); cudaFree(ctx->fo_sq);
    for (auto* p : ctx->d_gstack) cudaFree(p);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
    for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->evb) if (e) cudaEventDestroy(e);
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return OUC_OK;
}

int ouc_set_step_kernel(ouc_ctx* ctx, int seg_rows) {
    if (!ctx) return OUC_EINVAL;
    if (seg_rows != 0 && seg_rows != OUC_STEP_TILE_QUEUE && (seg_rows < 16 || seg_rows % 16 != 0))
        return fail(ctx, OUC_EINVAL, "segment rows must be 0 (tiles), OUC_STEP_TILE_QUEUE or a positive multiple of 16");
    if (seg_rows == ctx->seg_rows) return OUC_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    // captured time loops hold the old launch configuration
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
    ctx->seg_rows = seg_rows;
    return OUC_OK;
}

int ouc_time_step_kernels(ouc_ctx* ctx, int n, int reps, float* ms) {
    if (!ctx || !ms || n < 1 || n > ctx->batch || reps < 1) return OUC_EINVAL;
    if (!ctx->strips || ctx->nt < 4) return fail(ctx, OUC_ESTATE, "run an RTM batch of these shots first");
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    int rc;
    const int t = ctx->nt / 2;
    Side s = ctx->src, r = ctx->rcv;
    StepArgs a = base_args(ctx);
    a.record = 0;
    a.save = ctx->cfg.snapshot_every == 0;
    StepArgs ar = rcv_args(ctx), as = rec_args(ctx);
    const bool exact = ctx->cfg.strip_level == OUC_STRIP_EXACT;
    for (int kind = 0; kind < 3; ++kind) {
        for (int k = 0; k < reps + 1; ++k) {   // one warm-up launch, then `reps` timed
            if (k == 1) CK(cudaEventRecord(ctx->ev[0], ctx->stream));
            if (kind == 0) rc = fwd_step(ctx, a, s, n, t);
            else if (kind == 1) rc = rcv_step(ctx, ar, r, n, t);
            else rc = rec_step(ctx, as, s, r, n, t, exact, true);
            if (rc) return rc;
        }
        CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ms[kind] = elapsed(ctx->ev[0], ctx->ev[1]) / reps;
    }
    return check_status(ctx);
}

int ouc_debug_copy_stall(ouc_ctx* ctx, int on) {
    if (!ctx || (on != 0 && on != 1)) return OUC_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
    ctx->copy_stall = on != 0;
    return OUC_OK;
}

int ouc_get_step_kernel(const ouc_ctx* ctx, int* seg_rows) {
    if (!ctx || !seg_rows) return OUC_EINVAL;
    *seg_rows = ctx->seg_rows;
    return OUC_OK;
}

int ouc_dims(const ouc_ctx* ctx, int* X, int* Z) {
    if (!ctx) return OUC_EINVAL;
    if (X) *X = ctx->X;
    if (Z) *Z = ctx->Z;
    return OUC_OK;
}

void* ouc_stream(const ouc_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int ouc_last_timing(const ouc_ctx* ctx, ouc_timing* t) {
    if (!ctx || !t) return OUC_EINVAL;
    *t = ctx->timing;
    return OUC_OK;
}

size_t ouc_device_bytes(const ouc_ctx* ctx) { return ctx ? ctx->bytes : 0; }

static int forward_impl(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, float* gx, float* gz,
                        float* fields, bool host) {
    if (!ctx) return OUC_EINVAL;
    int rc = check_shot(ctx, shot);
    if (rc) return rc;
    if (!wavelet) return fail(ctx, OUC_EINVAL, "wavelet is NULL");
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;   // whole-shot calls overwrite any stepped state
    ctx->timing = ouc_timing{};
    const float* d_w = wavelet;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    if (host) {
        CK(cudaMemcpyAsync(ctx->d_wavelet, wavelet, (size_t)ctx->nt * 4, cudaMemcpyHostToDevice, ctx->stream));
        d_w = ctx->d_wavelet;
    }
    if ((rc = upload_desc(ctx, 1, shot, d_w))) return rc;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    if ((rc = run_forward(ctx, 1, gx || gz, false))) return rc;
    // runtime stability check: the recorded gathers (the receiver row of
    // every step) and the final level must be finite
    launch_finite_check(ctx->gather(0, 0), 2 * (size_t)ctx->nt * ctx->X, ctx->d_status, ctx->stream);
    launch_finite_check(ctx->src.now[0] - (size_t)kGX * ctx->pitch - kZOFF, ctx->fstride, ctx->d_status, ctx->stream);
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    if (gx && (rc = gather_out(ctx, ctx->gather(0, 0), gx, host))) return rc;
    if (gz && (rc = gather_out(ctx, ctx->gather(0, 1), gz, host))) return rc;
    if (fields && host) {
        const float* f[4] = {ctx->src.now[0], ctx->src.now[1], ctx->src.now[2], ctx->src.now[3]};
        launch_pack_fields(f, 4, ctx->X, ctx->Z, ctx->pitch, ctx->staging, ctx->stream);
        const size_t C = (size_t)ctx->X * ctx->Z;
        CK(cudaMemcpyAsync(fields + 2 * C, ctx->staging, 4 * C * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if ((rc = check_status(ctx))) return rc;
    if (fields && host) {
        const size_t C = (size_t)ctx->X * ctx->Z;
        for (size_t k = 0; k < C; ++k) {
            fields[k] = fields[2 * C + k] + fields[4 * C + k];       // Ux = Px + Sx
            fields[C + k] = fields[3 * C + k] + fields[5 * C + k];   // Uz = Pz + Sz
        }
    }
    ctx->timing.forward_ms = elapsed(ctx->ev[1], ctx->ev[2]);
    ctx->timing.copy_ms = elapsed(ctx->ev[0], ctx->ev[1]) + elapsed(ctx->ev[2], ctx->ev[3]);
    return OUC_OK;
}

int ouc_forward(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, float* gx, float* gz, float* fields) {
    return forward_impl(ctx, shot, wavelet, gx, gz, fields, true);
}

int ouc_forward_dev(ouc_ctx* ctx, const ouc_shot* shot, const float* d_wavelet, float* d_gx, float* d_gz) {
    return forward_impl(ctx, shot, d_wavelet, d_gx, d_gz, nullptr, false);
}

// One group of n <= batch shots.
static int rtm_group(ouc_ctx* ctx, int n, const ouc_shot* shots, const float* d_w, const float* const* rx,
                     const float* const* rz, float* const* ipp, float* const* ips, bool host) {
    int rc;
    const bool self_records = rx == nullptr;
    const bool snap = ctx->cfg.snapshot_every > 0;
    if ((rc = upload_desc(ctx, n, shots, d_w))) return rc;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    if ((rc = run_forward(ctx, n, self_records, !snap, snap))) return rc;
    for (int b = 0; b < n && !self_records; ++b) {
        if (!rx[b] || !rz[b]) return fail(ctx, OUC_EINVAL, "record pointer missing for a shot");
        if ((rc = gather_in(ctx, rx[b], ctx->gather(b, 0), host))) return rc;
        if ((rc = gather_in(ctx, rz[b], ctx->gather(b, 1), host))) return rc;
    }
    for (int b = 0; b < n; ++b) {
        if (!shots[b].mute) continue;
        const int sx = shots[b].sx + ctx->L, sz = shots[b].sz + ctx->L, rzz = shots[b].rz + ctx->L;
        const float v = ctx->vp_host[(size_t)sx * ctx->Z + rzz];   // Vp at (Sx, Z_receive), PS:1645
        launch_mute(ctx->gather(b, 0), ctx->gather(b, 1), ctx->X, ctx->nt, sx, sz, rzz, shots[b].t0, ctx->cfg.dt,
                    ctx->cfg.dx, v, ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    const bool theta = shots[0].src_type == OUC_SRC_THETA;
    for (int b = 1; b < n; ++b)
        if ((shots[b].src_type == OUC_SRC_THETA) != theta) return fail(ctx, OUC_EINVAL, "mixed source types in a batch");
    rc = snap ? run_backward_snap(ctx, n) : run_backward(ctx, n, ctx->cfg.strip_level == OUC_STRIP_EXACT, theta);
    if (rc) return rc;
    // runtime stability check: the modelled gathers and the imaging
    // accumulators (source illumination and both correlations) must be finite
    if (self_records) launch_finite_check(ctx->gather(0, 0), 2 * (size_t)ctx->nt * ctx->X * n, ctx->d_status, ctx->stream);
    for (int b = 0; b < n; ++b)
        launch_finite_check(ctx->acc[0] - (size_t)kGX * ctx->pitch - kZOFF + (size_t)b * ctx->shot_stride,
                            3 * ctx->fstride, ctx->d_status, ctx->stream);
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    if ((rc = finalize(ctx, n))) return rc;
    if (ctx->cfg.gradient) {
        GradStackArgs gs;
        gs.X = ctx->X; gs.Z = ctx->Z; gs.pitch = ctx->pitch; gs.L = ctx->L; gs.nshots = n;
        for (int k = 0; k < 3; ++k) {
            gs.g[k] = ctx->grad + (size_t)k * ctx->fstride + (size_t)kGX * ctx->pitch + kZOFF;
            gs.stack[k] = ctx->d_gstack[k];
        }
        gs.grad_stride = 3 * ctx->fstride;
        launch_grad_stack(gs, ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    const cudaMemcpyKind kind = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    for (int b = 0; b < n; ++b) {
        if (ipp && ipp[b]) CK(cudaMemcpyAsync(ipp[b], ctx->d_img + (size_t)(2 * b) * ni, ni * 4, kind, ctx->stream));
        if (ips && ips[b]) CK(cudaMemcpyAsync(ips[b], ctx->d_img + (size_t)(2 * b + 1) * ni, ni * 4, kind, ctx->stream));
    }
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if ((rc = check_status(ctx))) return rc;
    ctx->timing.forward_ms += elapsed(ctx->ev[0], ctx->ev[1]);
    ctx->timing.backward_ms += elapsed(ctx->ev[1], ctx->ev[2]);
    ctx->timing.finalize_ms += elapsed(ctx->ev[2], ctx->ev[3]);
    return OUC_OK;
}

static int rtm_batch_impl(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const float* wavelet,
                          const float* const* rx, const float* const* rz, float* const* ipp, float* const* ips,
                          bool host) {
    if (!ctx) return OUC_EINVAL;
    if (nshots < 1 || !shots) return fail(ctx, OUC_EINVAL, "no shots");
    if (!wavelet) return fail(ctx, OUC_EINVAL, "wavelet is NULL");
    if ((rx == nullptr) != (rz == nullptr)) return fail(ctx, OUC_EINVAL, "give both record components or neither");
    int rc;
    for (int b = 0; b < nshots; ++b)
        if ((rc = check_shot(ctx, &shots[b]))) return rc;
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;   // whole-shot calls overwrite any stepped state
    if ((rc = ctx->cfg.snapshot_every > 0 ? ensure_snaps(ctx) : ensure_strips(ctx))) return rc;
    if (ctx->cfg.gradient && (rc = ensure_grad(ctx))) return rc;
    ctx->timing = ouc_timing{};
    const float* d_w = wavelet;
    if (host) {
        CK(cudaMemcpyAsync(ctx->d_wavelet, wavelet, (size_t)ctx->nt * 4, cudaMemcpyHostToDevice, ctx->stream));
        d_w = ctx->d_wavelet;
    }
    for (int s0 = 0; s0 < nshots; s0 += ctx->run_batch) {
        const int n = std::min(ctx->run_batch, nshots - s0);
        rc = rtm_group(ctx, n, shots + s0, d_w, rx ? rx + s0 : nullptr, rz ? rz + s0 : nullptr, ipp ? ipp + s0 : nullptr,
                       ips ? ips + s0 : nullptr, host);
        if (rc) return rc;
    }
    return OUC_OK;
}

int ouc_rtm_shot(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, const float* rx, const float* rz,
                 float* img_pp, float* img_ps) {
    return rtm_batch_impl(ctx, 1, shot, wavelet, rx ? &rx : nullptr, rz ? &rz : nullptr, &img_pp, &img_ps, true);
}

int ouc_rtm_shot_dev(ouc_ctx* ctx, const ouc_shot* shot, const float* d_wavelet, const float* d_rx, const float* d_rz,
                     float* d_img_pp, float* d_img_ps) {
    return rtm_batch_impl(ctx, 1, shot, d_wavelet, d_rx ? &d_rx : nullptr, d_rz ? &d_rz : nullptr, &d_img_pp,
                          &d_img_ps, false);
}

int ouc_rtm_batch(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const float* wavelet, const float* const* rx,
                  const float* const* rz, float* const* ipp, float* const* ips) {
    return rtm_batch_impl(ctx, nshots, shots, wavelet, rx, rz, ipp, ips, true);
}

int ouc_rtm_batch_dev(ouc_ctx* ctx, int nshots, const ouc_shot* shots, const float* d_wavelet, const float* const* rx,
                      const float* const* rz, float* const* ipp, float* const* ips) {
    return rtm_batch_impl(ctx, nshots, shots, d_wavelet, rx, rz, ipp, ips, false);
}

int ouc_stack(ouc_ctx* ctx, double* pp, double* ps, double* illum, int reset) {
    if (!ctx) return OUC_EINVAL;
    cudaSetDevice(ctx->device);
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    double* outs[3] = {pp, ps, illum};
    for (int k = 0; k < 3; ++k)
        if (outs[k]) CK(cudaMemcpyAsync(outs[k], ctx->d_stack[k], ni * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (reset)
        for (int k = 0; k < 3; ++k) CK(cudaMemsetAsync(ctx->d_stack[k], 0, ni * 8, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OUC_OK;
}

int ouc_gradient(ouc_ctx* ctx, double* g_vp, double* g_vs, double* illum, int reset) {
    if (!ctx) return OUC_EINVAL;
    if (!ctx->cfg.gradient) return fail(ctx, OUC_ESTATE, "the context was created without gradient = 1");
    if (!ctx->grad) return fail(ctx, OUC_ESTATE, "no RTM shot has run yet");
    cudaSetDevice(ctx->device);
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    double* out[3] = {g_vp, g_vs, illum};
    for (int k = 0; k < 3; ++k)
        if (out[k]) CK(cudaMemcpyAsync(out[k], ctx->d_gstack[k], ni * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (reset)
        for (int k = 0; k < 3; ++k) CK(cudaMemsetAsync(ctx->d_gstack[k], 0, ni * 8, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OUC_OK;
}

int ouc_stack_dev(ouc_ctx* ctx, const double** pp, const double** ps, const double** illum) {
    if (!ctx) return OUC_EINVAL;
    if (pp) *pp = ctx->d_stack[0];
    if (ps) *ps = ctx->d_stack[1];
    if (illum) *illum = ctx->d_stack[2];
    return OUC_OK;
}

// ---- step-level interface -------------------------------------------------

static int step_order(ouc_ctx* ctx, int phase, int t) {
    if (ctx->step_phase != phase || t != ctx->step_t) {
        static const char* names[] = {"ouc_step_begin", "ouc_step_forward", "ouc_step_receiver",
                                      "ouc_step_reconstruct", "ouc_image_finalize"};
        const char* want = names[ctx->step_phase];
        return fail(ctx, OUC_ESTATE, std::string("step call out of order: expected ") + want +
                                         (ctx->step_phase == ouc_ctx::kIdle || ctx->step_phase == ouc_ctx::kFinalize
                                              ? std::string()
                                              : " at t = " + std::to_string(ctx->step_t)));
    }
    cudaSetDevice(ctx->device);
    return OUC_OK;
}

int ouc_step_begin(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, const float* rec_vx,
                   const float* rec_vz) {
    if (!ctx) return OUC_EINVAL;
    int rc = check_shot(ctx, shot);
    if (rc) return rc;
    if (!wavelet) return fail(ctx, OUC_EINVAL, "wavelet is NULL");
    if ((rec_vx == nullptr) != (rec_vz == nullptr)) return fail(ctx, OUC_EINVAL, "give both record components or neither");
    if (ctx->cfg.snapshot_every > 0)
        return fail(ctx, OUC_EINVAL, "the step-level calls follow the reconstruction form (snapshot_every = 0)");
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    if ((rc = ensure_strips(ctx))) return rc;
    ctx->timing = ouc_timing{};
    CK(cudaMemcpyAsync(ctx->d_wavelet, wavelet, (size_t)ctx->nt * 4, cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = upload_desc(ctx, 1, shot, ctx->d_wavelet))) return rc;
    if ((rc = zero_side(ctx, 1, 0, false)) || (rc = zero_side(ctx, 1, 1, true))) return rc;
    if (rec_vx) {
        if ((rc = gather_in(ctx, rec_vx, ctx->gather(0, 0), true))) return rc;
        if ((rc = gather_in(ctx, rec_vz, ctx->gather(0, 1), true))) return rc;
    }
    ctx->step_shot = *shot;
    ctx->step_fwd = base_args(ctx);
    ctx->step_fwd.record = rec_vx == nullptr;
    ctx->step_fwd.save = 1;
    ctx->step_rcv = rcv_args(ctx);
    ctx->step_rec = rec_args(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->step_phase = ouc_ctx::kForward;
    ctx->step_t = 0;
    return OUC_OK;
}

int ouc_step_forward(ouc_ctx* ctx, int t) {
    if (!ctx) return OUC_EINVAL;
    int rc = step_order(ctx, ouc_ctx::kForward, t);
    if (rc || (rc = fwd_step(ctx, ctx->step_fwd, ctx->src, 1, t))) return rc;
    CK(cudaGetLastError());
    if (++ctx->step_t < ctx->nt) return OUC_OK;
    // forward done: mute the records as the whole-shot path does (PS:2296-2297)
    const ouc_shot& sh = ctx->step_shot;
    if (sh.mute) {
        const int sx = sh.sx + ctx->L, sz = sh.sz + ctx->L, rzz = sh.rz + ctx->L;
        launch_mute(ctx->gather(0, 0), ctx->gather(0, 1), ctx->X, ctx->nt, sx, sz, rzz, sh.t0, ctx->cfg.dt,
                    ctx->cfg.dx, ctx->vp_host[(size_t)sx * ctx->Z + rzz], ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    ctx->step_phase = ouc_ctx::kReceiver;
    ctx->step_t = ctx->nt - 1;
    return OUC_OK;
}

int ouc_step_receiver(ouc_ctx* ctx, int t) {
    if (!ctx) return OUC_EINVAL;
    int rc = step_order(ctx, ouc_ctx::kReceiver, t);
    if (rc || (rc = rcv_step(ctx, ctx->step_rcv, ctx->rcv, 1, t))) return rc;
    CK(cudaGetLastError());
    ctx->step_phase = ouc_ctx::kReconstruct;
    return OUC_OK;
}

int ouc_step_reconstruct(ouc_ctx* ctx, int t) {
    if (!ctx) return OUC_EINVAL;
    int rc = step_order(ctx, ouc_ctx::kReconstruct, t);
    if (rc) return rc;
    rc = rec_step(ctx, ctx->step_rec, ctx->src, ctx->rcv, 1, t, ctx->cfg.strip_level == OUC_STRIP_EXACT,
                  ctx->step_shot.src_type == OUC_SRC_THETA);
    if (rc) return rc;
    CK(cudaGetLastError());
    if (--ctx->step_t >= 0) {
        ctx->step_phase = ouc_ctx::kReceiver;
    } else {
        ctx->step_phase = ouc_ctx::kFinalize;
        ctx->step_t = 0;
    }
    return OUC_OK;
}

int ouc_image_finalize(ouc_ctx* ctx, float* img_pp, float* img_ps) {
    if (!ctx) return OUC_EINVAL;
    int rc = step_order(ctx, ouc_ctx::kFinalize, 0);
    if (rc || (rc = finalize(ctx, 1))) return rc;
    const size_t ni = (size_t)ctx->nx * ctx->nz;
    if (img_pp) CK(cudaMemcpyAsync(img_pp, ctx->d_img, ni * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (img_ps) CK(cudaMemcpyAsync(img_ps, ctx->d_img + ni, ni * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->step_phase = ouc_ctx::kIdle;
    return OUC_OK;
}

int ouc_step_fields(ouc_ctx* ctx, int side, float* fields) {
    if (!ctx) return OUC_EINVAL;
    if (!fields || (side != 0 && side != 1)) return fail(ctx, OUC_EINVAL, "fields is NULL or side is not 0/1");
    if (ctx->step_phase == ouc_ctx::kIdle) return fail(ctx, OUC_ESTATE, "no shot is being stepped");
    cudaSetDevice(ctx->device);
    const Side& s = side == 0 ? ctx->src : ctx->rcv;
    const float* f[4] = {s.now[0], s.now[1], s.now[2], s.now[3]};
    launch_pack_fields(f, 4, ctx->X, ctx->Z, ctx->pitch, ctx->staging, ctx->stream);
    const size_t C = (size_t)ctx->X * ctx->Z;
    CK(cudaMemcpyAsync(fields + 2 * C, ctx->staging, 4 * C * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t k = 0; k < C; ++k) {
        fields[k] = fields[2 * C + k] + fields[4 * C + k];       // Ux = Px + Sx (PS:302)
        fields[C + k] = fields[3 * C + k] + fields[5 * C + k];   // Uz = Pz + Sz (PS:303)
    }
    return OUC_OK;
}

}  // extern "C"
