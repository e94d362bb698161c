// First-order velocity-stress forward modeling (ouc_forward_fo): the scheme
// of the reference's stress (PS:487-560) and velocity (PS:390-486) kernels,
// which its main() never calls, as one fused sm_100a launch per time step.
//
// State: the P/S velocity parts (Vpx, Vpz, Vsx, Vsz) and eight split stresses
// (theta_x, theta_z, omega_x, omega_z and the four Q fields), each
// ping-ponged so that the halo reads of one step never meet its writes.  One
// 32 x 64 tile per CTA, in three phases like the second-order step kernel:
//   1. U = P + S velocity over the tile and a 2N halo into shared memory;
//   2. the stress update over the tile and an N halo (four staggered velocity
//      derivatives, the split-field damping (1 - dt a/2)/(1 + dt a/2), the
//      source on theta), own cells written out, theta/omega/Q kept on chip;
//   3. the velocity update of the own cells from eight stress derivatives,
//      U = P + S, the receiver row recorded after the update.
// Derivatives use the rounding-exact helpers of fd_step.cuh; the damping
// factors and updates are the reference's expressions verbatim (double
// literals, so double arithmetic rounded once to float), powf(v, 2) as
// there, so that the compiler contracts them as it does the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/ouc.h"
#include "ctx.h"
#include "fd_step.cuh"

namespace ouc {
namespace fo {

struct FoArgs {
    int X, Z, pitch, tiles_z, t, nt;
    int sx, sz, rz;                  // padded source cell and receiver row
    float a[6];
    float dx, dz, dt, rdx, rdz;
    const float* vold[4];            // Vpx Vpz Vsx Vsz at the old half level
    float* vnew[4];
    const float* sold[8];            // theta_x theta_z omega_x omega_z Qxx Qxz Qzx Qzz
    float* snew[8];
    const float* vp2;                // powf(Vp, 2), powf(Vs, 2) (k_squares), damping x, z
    const float* vs2;
    const float* ax;
    const float* az;
    const float* wavelet;            // source samples, or null (back-propagation)
    float* rec_x;                    // gather row t (time-major), or null
    float* rec_z;
    const float* inj_x;              // records injected into U at the receiver
    const float* inj_z;              // row on [L, X-L) (row t), or null
    int L;
};

// split-field stress update, the reference's expression (PS:547-556)
__device__ __forceinline__ float stress_upd(float damp, float dt, float term, float old) {
    return (1.0 / (1.0 + 0.5 * dt * damp)) * (term + (1.0 - 0.5 * dt * damp) * old);
}
// velocity update, the reference's expression (PS:471-474)
__device__ __forceinline__ float vel_upd(float damp, float dt, float old, float sum) {
    return (1.0 / (1.0 + 0.5 * dt * damp)) * ((1 - 0.5 * dt * damp) * old + dt * sum);
}
// Both updates where the damping is 0 (the interior): the factors are exactly
// 1, and the double sum of two floats rounded to float is their float sum
// (53 >= 2*24 + 2: the double rounding is innocuous), so the result is one
// float addition -- bit-identical, without the double arithmetic.
__device__ __forceinline__ bool undamped4(const float4& ax, const float4& az) {
    return ax.x == 0.f && ax.y == 0.f && ax.z == 0.f && ax.w == 0.f && az.x == 0.f && az.y == 0.f && az.z == 0.f &&
           az.w == 0.f;
}

// powf(v, 2) of the model once per call, as the kernels evaluate it per cell
// (PS:547); guard cells hold 0.
__global__ void k_squares(const float* __restrict__ vp, const float* __restrict__ vs, float* vp2, float* vs2,
                          size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        vp2[k] = powf(vp[k], 2);
        vs2[k] = powf(vs[k], 2);
    }
}

template <int N>
__global__ void __launch_bounds__(kThreads, 2) k_fo(const FoArgs p) {
    using G = TileGeo<N>;
    constexpr int TX = G::TX, TZ = G::TZ, SHX = G::SHX, HS = G::HS, HU = G::HU, UC = G::UC, SC = G::SC;
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    float* sUx = sm + G::oUx;
    float* sUz = sm + G::oUz;
    float* sTh = sm + G::oTh;
    float* sOm = sm + G::oOm;
    float* sQxz = sm + G::oQxz;
    float* sQzz = sm + G::oQzz;
    float* sQxx = sm + G::oQxx;
    float* sQzx = sm + G::oQzx;
    const int tid = threadIdx.x;
    const int P = p.pitch;
    const int tz = blockIdx.x % p.tiles_z, tx = blockIdx.x / p.tiles_z;
    const int x0 = tx * TX, z0 = tz * TZ;
    float a[N];
#pragma unroll
    for (int k = 0; k < N; ++k) a[k] = p.a[k];
    const Div dvx = make_div(p.dx, p.rdx), dvz = make_div(p.dz, p.rdz);
    const float dt = p.dt;
    const int ux_i0 = x0 - SHX - N, ux_j0 = z0 - HU;

    // ---- phase 1: U = P + S velocity over the tile and a 2N halo ----------
    for (int idx = tid; idx < G::UR * (UC / 4); idx += kThreads) {
        const int r = idx / (UC / 4), c4 = idx - r * (UC / 4);
        const int g = (ux_i0 + r) * P + (ux_j0 + 4 * c4);
        float4 ux = add4(ld4(p.vold[0] + g), ld4(p.vold[2] + g));   // Vx = Vpx + Vsx
        float4 uz = add4(ld4(p.vold[1] + g), ld4(p.vold[3] + g));
        const int gi = ux_i0 + r, gj = ux_j0 + 4 * c4;
        if (p.inj_x && p.rz >= gj && p.rz < gj + 4 && gi >= p.L && gi < p.X - p.L) {
            // load_record (PS:1472-1481): U at the receiver row replaced by
            // the records before the stress update reads it
            set_comp(ux, p.rz - gj, p.inj_x[gi]);
            set_comp(uz, p.rz - gj, p.inj_z[gi]);
        }
        st4(sUx + r * UC + 4 * c4, ux);
        st4(sUz + r * UC + 4 * c4, uz);
    }
    __syncthreads();

    // ---- phase 2: stresses on the tile plus an N halo ----------------------
    if (tid < G::itemsA + G::itemsB) {
        int r0, c;
        const bool groupA = tid < G::itemsA;
        if (groupA) {
            r0 = -SHX + 4 * (tid / (TZ / 4));
            c = 4 * (tid % (TZ / 4));
        } else {
            const int k = tid - G::itemsA;
            r0 = 4 * (k / (2 * HS / 4));
            const int cc = k % (2 * HS / 4);
            c = cc < HS / 4 ? -HS + 4 * cc : TZ + 4 * (cc - HS / 4);
        }
        const float* ux0 = sUx + (r0 + SHX + N) * UC + (c + HU);
        const float* uz0 = sUz + (r0 + SHX + N) * UC + (c + HU);
        float4 exx[4], ezx[4];
        dx4<N, 4, false>(ux0, UC, a, dvx, exx);   // dvxdx = D-x Vx
        dx4<N, 4, true>(uz0, UC, a, dvx, ezx);    // dvzdx = D+x Vz
        const bool ownc = c >= 0 && c < TZ;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r0 + q, gi = x0 + r, gjb = z0 + c;
            const float4 exz = dz4<N, true>(ux0 + q * UC, a, dvz);    // dvxdz = D+z Vx
            const float4 ezz = dz4<N, false>(uz0 + q * UC, a, dvz);   // dvzdz = D-z Vz
            const int g = gi * P + gjb;
            const float4 vp2v = ld4(p.vp2 + g), vs2v = ld4(p.vs2 + g), axv = ld4(p.ax + g), azv = ld4(p.az + g);
            float4 so[8], sn[8];
#pragma unroll
            for (int f = 0; f < 8; ++f) so[f] = ld4(p.sold[f] + g);
            const bool row_live = gi >= N && gi < p.X - N;
            const bool flat = undamped4(axv, azv);
            float th[4], om[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int gj = gjb + k;
                const bool live = row_live && gj >= N && gj < p.Z - N;
                const float cp = __fmul_rn(dt, comp(vp2v, k)), cs = __fmul_rn(dt, comp(vs2v, k));
                const float dxx = comp(exx[q], k), dzz = comp(ezz, k), dxz = comp(exz, k), dzx = comp(ezx[q], k);
                // dt Vp^2 d, dt Vs^2 d and -dt Vs^2 d, each rounded as the reference's float products
                float term[8];
                term[0] = __fmul_rn(cp, dxx);    // theta_x
                term[1] = __fmul_rn(cp, dzz);    // theta_z
                term[2] = __fmul_rn(-cs, dzx);   // omega_x
                term[3] = __fmul_rn(cs, dxz);    // omega_z
                term[4] = __fmul_rn(cs, dxx);    // Qxx (duxdx)
                term[5] = __fmul_rn(cs, dxz);    // Qxz (duxdz)
                term[6] = __fmul_rn(cs, dzx);    // Qzx (duzdx)
                term[7] = __fmul_rn(cs, dzz);    // Qzz (duzdz)
                float v[8];
                if (flat) {
#pragma unroll
                    for (int f = 0; f < 8; ++f) v[f] = __fadd_rn(term[f], comp(so[f], k));
                } else {
                    const float dax = comp(axv, k), daz = comp(azv, k);
#pragma unroll
                    for (int f = 0; f < 8; ++f) v[f] = stress_upd((f & 1) ? daz : dax, dt, term[f], comp(so[f], k));
                }
#pragma unroll
                for (int f = 0; f < 8; ++f) {
                    if (!live) v[f] = 0.f;   // the reference never updates these cells
                    set_comp(sn[f], k, v[f]);
                }
                const float s = (p.wavelet && live && gi == p.sx && gj == p.sz) ? p.wavelet[p.t] : 0.f;
                th[k] = v[0] + v[1] + s;   // PS:557
                om[k] = v[2] + v[3];
            }
            const bool own = ownc && r >= 0 && r < TX;
            if (own) {
#pragma unroll
                for (int f = 0; f < 8; ++f) st4(p.snew[f] + g, sn[f]);
            }
            const int sr = r + SHX, scol = c + HS;
            st4(sTh + sr * SC + scol, make_float4(th[0], th[1], th[2], th[3]));
            st4(sOm + sr * SC + scol, make_float4(om[0], om[1], om[2], om[3]));
            if (groupA) {
                st4(sQxz + sr * TZ + c, sn[5]);
                st4(sQzz + sr * TZ + c, sn[7]);
            }
            if (r >= 0 && r < TX) {
                st4(sQxx + r * SC + scol, sn[4]);
                st4(sQzx + r * SC + scol, sn[6]);
            }
        }
    }
    __syncthreads();

    // ---- phase 3: velocities of the own cells (2 rows x 4 columns) ---------
    {
        const int rr = 2 * (tid / (TZ / 4));
        const int c = 4 * (tid % (TZ / 4));
        const int scol = c + HS;
#pragma unroll 1
        for (int q = 0; q < 2; ++q) {
            const int r = rr + q, gi = x0 + r;
            float4 txv[1], wxv[1], dB[1], dE[1];
            dx4<N, 1, true>(sTh + (r + SHX) * SC + scol, SC, a, dvx, txv);    // dthetadx = D+x theta
            dx4<N, 1, false>(sOm + (r + SHX) * SC + scol, SC, a, dvx, wxv);   // domegadx = D-x omega
            dx4<N, 1, false>(sQxz + (r + SHX) * TZ + c, TZ, a, dvx, dB);      // dux_zdx = D-x Qxz
            dx4<N, 1, true>(sQzz + (r + SHX) * TZ + c, TZ, a, dvx, dE);       // duz_zdx = D+x Qzz
            const float4 tzv = dz4<N, true>(sTh + (r + SHX) * SC + scol, a, dvz);   // dthetadz
            const float4 wzv = dz4<N, false>(sOm + (r + SHX) * SC + scol, a, dvz);  // domegadz
            const float4 dA = dz4<N, true>(sQxx + r * SC + scol, a, dvz);           // dux_xdz = D+z Qxx
            const float4 dC = dz4<N, false>(sQzx + r * SC + scol, a, dvz);          // duz_xdz = D-z Qzx
            const int g = gi * P + (z0 + c);
            const float4 axv = ld4(p.ax + g), azv = ld4(p.az + g);
            const float4 opx = ld4(p.vold[0] + g), opz = ld4(p.vold[1] + g);
            const float4 osx = ld4(p.vold[2] + g), osz = ld4(p.vold[3] + g);
            float4 npx, npz, nsx, nsz;
            const bool row_live = gi >= N && gi < p.X - N;
            const bool flat = undamped4(axv, azv);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int gj = z0 + c + k;
                const bool live = row_live && gj >= N && gj < p.Z - N;
                const float C = comp(dC, k), E = comp(dE[0], k), A = comp(dA, k), B = comp(dB[0], k);
                const float sum_px = __fsub_rn(__fadd_rn(comp(txv[0], k), C), E);
                const float sum_pz = __fsub_rn(__fadd_rn(comp(tzv, k), B), A);
                const float sum_sx = __fsub_rn(__fadd_rn(comp(wzv, k), C), E);
                const float sum_sz = __fsub_rn(__fadd_rn(-comp(wxv[0], k), B), A);
                float vpx, vpz, vsx, vsz;
                if (flat) {
                    vpx = __fadd_rn(comp(opx, k), __fmul_rn(dt, sum_px));
                    vpz = __fadd_rn(comp(opz, k), __fmul_rn(dt, sum_pz));
                    vsx = __fadd_rn(comp(osx, k), __fmul_rn(dt, sum_sx));
                    vsz = __fadd_rn(comp(osz, k), __fmul_rn(dt, sum_sz));
                } else {
                    const float dax = comp(axv, k), daz = comp(azv, k);
                    vpx = vel_upd(dax, dt, comp(opx, k), sum_px);
                    vpz = vel_upd(daz, dt, comp(opz, k), sum_pz);
                    vsx = vel_upd(dax, dt, comp(osx, k), sum_sx);
                    vsz = vel_upd(daz, dt, comp(osz, k), sum_sz);
                }
                if (!live) vpx = vpz = vsx = vsz = 0.f;
                set_comp(npx, k, vpx); set_comp(npz, k, vpz); set_comp(nsx, k, vsx); set_comp(nsz, k, vsz);
            }
            st4(p.vnew[0] + g, npx); st4(p.vnew[1] + g, npz);
            st4(p.vnew[2] + g, nsx); st4(p.vnew[3] + g, nsz);
            if (p.rec_x && p.rz >= z0 + c && p.rz < z0 + c + 4 && gi < p.X) {
                const int k = p.rz - z0 - c;   // post-update value at the receiver row
                p.rec_x[gi] = comp(npx, k) + comp(nsx, k);
                p.rec_z[gi] = comp(npz, k) + comp(nsz, k);
            }
        }
    }
}

// The shared-memory opt-in is a per-device attribute: set on the current
// device before every loop (fo_run), not once per process.
template <int N>
cudaError_t configure() {
    return cudaFuncSetAttribute(k_fo<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, TileGeo<N>::bytes);
}

template <int N>
void launch(const FoArgs& a, int tiles_x, cudaStream_t s) {
    k_fo<N><<<tiles_x * a.tiles_z, kThreads, TileGeo<N>::bytes, s>>>(a);
}

// Five-digit weights of the reference's first-order kernels (PS:405,
// PS:501): double literals converted to float, as a float array initialised
// from them; other half-orders use the context's weights.
constexpr float kFoWeights6[6] = {(float)1.2213e+0, (float)-9.6931e-2, (float)1.7448e-2,
                                  (float)-2.9673e-3, (float)3.5901e-4, (float)-2.1848e-5};

}  // namespace fo
}  // namespace ouc

using namespace ouc;
using namespace ouc::host;

namespace {

int fo_check(ouc_ctx* ctx, const ouc_shot* shot) {
    if (!ctx) return OUC_EINVAL;
    int rc = check_shot(ctx, shot);
    if (rc) return rc;
    if (shot->src_type != OUC_SRC_THETA) return fail(ctx, OUC_EINVAL, "the first-order scheme has the theta source only");
    if (ctx->cfg.density) return fail(ctx, OUC_EINVAL, "the first-order scheme is density-normalised");
    return OUC_OK;
}

// The first-order time loop on the source side's 24 fields (velocities
// now[4] / past[4], stresses fo[4] + o[0..3] / fn[4] + o[4..7], ping-ponged
// by step).  Forward: t = 0 .. nt-1 with the source and the record into the
// context's gathers.  Backward: t = nt-1 .. 0 injecting the context's
// gathers (row t) at the receiver row.  fields (host, 16*X*Z, or null): the
// final state; `theta_src` is the source sample theta carries at the source
// cell in the last step (0 backward).
int fo_run(ouc_ctx* ctx, const ouc_shot* shot, bool backward, float theta_src, float* fields) {
    int rc;
    const size_t C = (size_t)ctx->X * ctx->Z;
    if (!ctx->fo_sq) {
        if (cudaMalloc(&ctx->fo_sq, 2 * ctx->fstride * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            ctx->fo_sq = nullptr;
            return fail(ctx, OUC_ENOMEM, "cannot allocate the first-order model squares");
        }
        ctx->bytes += 2 * ctx->fstride * sizeof(float);
    }
    // raw field bases (guards included) of Vp, Vs (model fields 6, 7) and the squares
    fo::k_squares<<<4 * 148, 256, 0, ctx->stream>>>(ctx->model + 6 * ctx->fstride, ctx->model + 7 * ctx->fstride,
                                                    ctx->fo_sq, ctx->fo_sq + ctx->fstride, ctx->fstride);
    ctx->timing.kernel_launches += 1;
    const cudaError_t ce = ctx->N == 2 ? fo::configure<2>() : ctx->N == 5 ? fo::configure<5>() : fo::configure<6>();
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "first-order kernel configuration");
    if ((rc = zero_side(ctx, 1, 0, false))) return rc;
    const Side& s = ctx->src0;
    const float* vA[4] = {s.now[0], s.now[1], s.now[2], s.now[3]};
    float* vB[4] = {s.past[0], s.past[1], s.past[2], s.past[3]};
    float* sA[8] = {s.fo[0], s.fo[1], s.fo[2], s.fo[3], s.o[0], s.o[1], s.o[2], s.o[3]};
    float* sB[8] = {s.fn[0], s.fn[1], s.fn[2], s.fn[3], s.o[4], s.o[5], s.o[6], s.o[7]};
    fo::FoArgs a;
    memset(&a, 0, sizeof(a));
    a.X = ctx->X; a.Z = ctx->Z; a.pitch = ctx->pitch; a.tiles_z = ctx->tiles_z; a.nt = ctx->nt; a.L = ctx->L;
    a.sx = shot->sx + ctx->L; a.sz = shot->sz + ctx->L; a.rz = shot->rz + ctx->L;
    for (int k = 0; k < 6; ++k) a.a[k] = ctx->N == 6 ? fo::kFoWeights6[k] : ctx->a[k];
    a.dx = ctx->cfg.dx; a.dz = ctx->cfg.dz; a.dt = ctx->cfg.dt;
    a.rdx = 1.0f / ctx->cfg.dx; a.rdz = 1.0f / ctx->cfg.dz;
    a.vp2 = ctx->field(ctx->fo_sq, 0); a.vs2 = ctx->field(ctx->fo_sq, 1); a.ax = ctx->ax; a.az = ctx->az;
    a.wavelet = backward ? nullptr : ctx->d_wavelet;
    float* gx = ctx->gather(0, 0);
    float* gz = ctx->gather(0, 1);
    cudaEventRecord(ctx->ev[1], ctx->stream);
    for (int n = 0; n < ctx->nt; ++n) {
        const int t = backward ? ctx->nt - 1 - n : n;
        const bool even = (n & 1) == 0;
        for (int k = 0; k < 4; ++k) { a.vold[k] = even ? vA[k] : vB[k]; a.vnew[k] = even ? vB[k] : (float*)vA[k]; }
        for (int k = 0; k < 8; ++k) { a.sold[k] = even ? sA[k] : sB[k]; a.snew[k] = even ? sB[k] : sA[k]; }
        a.t = t;
        if (backward) {
            a.inj_x = gx + (size_t)t * ctx->X;
            a.inj_z = gz + (size_t)t * ctx->X;
        } else {
            a.rec_x = gx + (size_t)t * ctx->X;
            a.rec_z = gz + (size_t)t * ctx->X;
        }
        if (ctx->N == 2) fo::launch<2>(a, ctx->tiles_x, ctx->stream);
        else if (ctx->N == 5) fo::launch<5>(a, ctx->tiles_x, ctx->stream);
        else fo::launch<6>(a, ctx->tiles_x, ctx->stream);
        ctx->timing.kernel_launches += 1;
    }
    cudaEventRecord(ctx->ev[2], ctx->stream);
    const cudaError_t le = cudaGetLastError();   // launch-configuration errors are not reported by the sync
    if (le != cudaSuccess) return cuda_fail(ctx, le, "first-order step launch");
    if (fields) {
        // the newest level: written by the last step
        const bool last_even = ((ctx->nt - 1) & 1) == 0;
        const float* v[4];
        const float* st[8];
        for (int k = 0; k < 4; ++k) v[k] = last_even ? vB[k] : vA[k];
        for (int k = 0; k < 8; ++k) st[k] = last_even ? sB[k] : sA[k];
        // 16 host fields: Vx Vz Vpx Vpz Vsx Vsz theta omega Qzx Qzz Qxx Qxz theta_x theta_z omega_x omega_z
        const float* order[12] = {v[0], v[1], v[2], v[3], st[6], st[7], st[4], st[5], st[0], st[1], st[2], st[3]};
        const int dst[12] = {2, 3, 4, 5, 8, 9, 10, 11, 12, 13, 14, 15};
        for (int k = 0; k < 12; k += 4) {
            launch_pack_fields(order + k, 4, ctx->X, ctx->Z, ctx->pitch, ctx->staging, ctx->stream);
            for (int q = 0; q < 4; ++q)
                if (cudaMemcpyAsync(fields + (size_t)dst[k + q] * C, ctx->staging + (size_t)q * C, C * 4,
                                    cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
                    return fail(ctx, OUC_ECUDA, "field download failed");
            if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(ctx, OUC_ECUDA, "field download failed");
        }
    }
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "first-order time loop");
    if (fields) {
        // totals as the kernels form them: U = P + S, theta = theta_x + theta_z + s,
        // omega = omega_x + omega_z
        const size_t src_cell = (size_t)(shot->sx + ctx->L) * ctx->Z + (shot->sz + ctx->L);
        for (size_t k = 0; k < C; ++k) {
            const float sv = k == src_cell ? theta_src : 0.0f;
            fields[k] = fields[2 * C + k] + fields[4 * C + k];
            fields[C + k] = fields[3 * C + k] + fields[5 * C + k];
            fields[6 * C + k] = fields[12 * C + k] + fields[13 * C + k] + sv;
            fields[7 * C + k] = fields[14 * C + k] + fields[15 * C + k];
        }
    }
    (backward ? ctx->timing.backward_ms : ctx->timing.forward_ms) = elapsed(ctx->ev[1], ctx->ev[2]);
    return OUC_OK;
}

}  // namespace

extern "C" {

int ouc_forward_fo(ouc_ctx* ctx, const ouc_shot* shot, const float* wavelet, float* gather_vx, float* gather_vz,
                   float* fields) {
    int rc = fo_check(ctx, shot);
    if (rc) return rc;
    if (!wavelet) return fail(ctx, OUC_EINVAL, "wavelet is NULL");
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    ctx->timing = ouc_timing{};
    if (cudaMemcpyAsync(ctx->d_wavelet, wavelet, (size_t)ctx->nt * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return fail(ctx, OUC_ECUDA, "wavelet upload failed");
    if ((rc = fo_run(ctx, shot, false, wavelet[ctx->nt - 1], fields))) return rc;
    if (gather_vx && (rc = gather_out(ctx, ctx->gather(0, 0), gather_vx, true))) return rc;
    if (gather_vz && (rc = gather_out(ctx, ctx->gather(0, 1), gather_vz, true))) return rc;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "gather download");
    return OUC_OK;
}

int ouc_backward_fo(ouc_ctx* ctx, const ouc_shot* shot, const float* rec_vx, const float* rec_vz, float* fields) {
    int rc = fo_check(ctx, shot);
    if (rc) return rc;
    if (!rec_vx || !rec_vz) return fail(ctx, OUC_EINVAL, "records are NULL");
    cudaSetDevice(ctx->device);
    ctx->step_phase = ouc_ctx::kIdle;
    ctx->timing = ouc_timing{};
    if ((rc = gather_in(ctx, rec_vx, ctx->gather(0, 0), true))) return rc;
    if ((rc = gather_in(ctx, rec_vz, ctx->gather(0, 1), true))) return rc;
    return fo_run(ctx, shot, true, 0.0f, fields);
}

}  // extern "C"
