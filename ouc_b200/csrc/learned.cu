// Learned dispersion correction of a coarse run (include/ouc_corrector.h).
//
// A coarse context runs the same step kernel at half-order 2 on a grid of
// twice the spacing and twice the time step of a fine context (half-order 5).
// Coarse padded cell (ic, jc) sits where fine padded cell (2ic, 2jc) sits
// (the absorbing widths satisfy L_fine = 2 L_coarse), so the cell-centred
// quantities (theta) coincide; the displacement components are staggered by
// half a cell (Ux at (i + 1/2, j), Uz at (i, j + 1/2): the D- x-derivative of
// Ux lands on theta, PS:340-366), which on the coarse grid is one whole fine
// cell away from any fine Ux/Uz point.  The restriction operator therefore
// interpolates the staggered direction at the midpoint with the 4-point cubic
// weights (-1, 9, 9, -1) / 16 and samples the other direction.
//
// Every `every` coarse steps the network reads the coarse state and returns
// a correction of the displacement components Px, Pz, Sx, Sz at the current
// leapfrog level and a correction of their change over the last step; both
// are applied on the correction region, U^n += s_d c_U / G and
// U^(n-1) += (s_d c_U - s_v c_V) / G (G = kGain, a fixed output scale that
// keeps the training targets near unit size).  Predicting the change
// directly keeps the implied particle velocity accurate: two independent
// level corrections would carry errors of the displacement's size into a
// difference about 10x smaller.  The correction region is the interior less a
// band of kEdge cells along the absorbing layers and a disc of radius
// kSrcRadius around the source: there the coarse/fine mismatch comes from the
// absorbing boundary and the point source's near field, not from dispersion.
//
// The corrector works in the band the coarse grid resolves.  Over one
// interval the fine/coarse mismatch has most of its energy at wavenumbers
// where the coarse state has almost none (below ~7 points per wavelength,
// much of it unresolvable); fitting it would need large gains there, which
// the closed loop amplifies.  So the training target is the mismatch
// low-passed by S, the 5-point binomial filter (1 4 6 4 1)/16 along x and
// along z (response cos^4(pi k) per axis, k in cycles per cell), and the
// applied correction is S of the network output.
//
// Network input channels, per cell (OUC_CNN_IN = 10): the leapfrog state
//   0-3   Px, Pz, Sx, Sz at level n, / s_d
//   4-7   their change over the last step U^n - U^(n-1), / s_v
//   8     (Vp/Vs - 1.7) g,   9   (Vp dt / h - 0.5) g
// with g = |ch 4| + |ch 5| + |ch 6| + |ch 7| and s_d, s_v the largest |U| and
// |U^n - U^(n-1)| over the interior.  The correction of a linear scheme is a
// linear function of the whole state, so the network sees all of it; the model
// channels are gated by the local motion and the network is trained without
// biases, so a quiet region (all inputs zero) receives exactly zero correction.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ouc.h"
#include "../../include/ouc_corrector.h"
#include "ctx.h"

namespace ouc {
namespace learned {

constexpr int kIn = OUC_CNN_IN;
constexpr int kOut = OUC_CNN_OUT;
constexpr float kGain = 16.f;     // targets are kGain x the correction
constexpr int kEdge = 4;          // cells kept clear of the absorbing layers
constexpr int kSrcRadius = 6;     // cells kept clear around the source

struct Level4 {
    const float* f[4];   // Px Pz Sx Sz, pitched, cell (0, 0)
};
struct Mut4 {
    float* f[4];
};
struct Rect {
    int i0, i1, j0, j1;
};
// the correction region: a rectangle less a disc around the source (sx, sz)
struct Region {
    Rect r;
    int sx, sz;
    __device__ __forceinline__ bool in(int i, int j) const {
        const int di = i - sx, dj = j - sz;
        return i >= r.i0 && i < r.i1 && j >= r.j0 && j < r.j1 && di * di + dj * dj > kSrcRadius * kSrcRadius;
    }
};

// midpoint of b and c on the 4-point stencil a b c d
__device__ __forceinline__ float mid4(float a, float b, float c, float d) { return (9.f * (b + c) - (a + d)) * 0.0625f; }

__device__ __forceinline__ float ld(const float* f, int pitch, int i, int j) { return f[(ptrdiff_t)i * pitch + j]; }

// Largest |U^n| and |U^n - U^(n-1)| over the rectangle, as float bits.
__global__ void k_scales(Level4 now, Level4 past, int pitch, Rect r, unsigned* out) {
    const int w = r.j1 - r.j0, n = (r.i1 - r.i0) * w;
    float md = 0.f, mv = 0.f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = r.i0 + k / w, j = r.j0 + k % w;
        const ptrdiff_t g = (ptrdiff_t)i * pitch + j;
        const float ux = now.f[0][g] + now.f[2][g], uz = now.f[1][g] + now.f[3][g];
        const float vx = ux - (past.f[0][g] + past.f[2][g]), vz = uz - (past.f[1][g] + past.f[3][g]);
        md = fmaxf(md, fmaxf(fabsf(ux), fabsf(uz)));
        mv = fmaxf(mv, fmaxf(fabsf(vx), fabsf(vz)));
    }
    for (int o = 16; o > 0; o >>= 1) {
        md = fmaxf(md, __shfl_xor_sync(0xffffffffu, md, o));
        mv = fmaxf(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (md > 0.f) atomicMax(out, __float_as_uint(md));
        if (mv > 0.f) atomicMax(out + 1, __float_as_uint(mv));
    }
}

__device__ __forceinline__ float inv_or_zero(unsigned bits) {
    const float s = __uint_as_float(bits);
    return s > 0.f ? 1.f / s : 0.f;
}

// Network input [X][Z][OUC_CNN_IN] of the state (now, past); every cell of the padded grid.
__global__ void k_pack_input(Level4 now, Level4 past, const float* vp2, const float* vs2, int X, int Z, int pitch,
                             float courant, const unsigned* scale, float* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= Z) return;
    const float id = inv_or_zero(scale[0]), iv = inv_or_zero(scale[1]);
    const ptrdiff_t g = (ptrdiff_t)i * pitch + j;
    float* o = out + ((size_t)i * Z + j) * kIn;
    float gate = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float u = now.f[q][g], v = u - past.f[q][g];
        o[q] = u * id;
        o[4 + q] = v * iv;
        gate += fabsf(v * iv);
    }
    const float a = vp2[g], b = vs2[g];
    o[8] = b > 0.f ? (sqrtf(a / b) - 1.7f) * gate : 0.f;
    o[9] = (sqrtf(a) * courant - 0.5f) * gate;
}

// Correction on the region: U^n += s_d c[0..3] / G, U^(n-1) += (s_d c[0..3] - s_v c[4..7]) / G.
__global__ void k_apply(const float* corr, int Z, int pitch, Region rg, const unsigned* scale, Mut4 now, Mut4 past) {
    const int j = rg.r.j0 + blockIdx.x * blockDim.x + threadIdx.x, i = rg.r.i0 + blockIdx.y;
    if (j >= rg.r.j1 || !rg.in(i, j)) return;
    const float sd = __uint_as_float(scale[0]) / kGain, sv = __uint_as_float(scale[1]) / kGain;
    const float* c = corr + ((size_t)i * Z + j) * kOut;
    const ptrdiff_t g = (ptrdiff_t)i * pitch + j;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float du = c[q] * sd;
        now.f[q][g] += du;
        past.f[q][g] += du - c[4 + q] * sv;
    }
}

// Noise of relative size (nd, nv) added to a state on the region (training
// input augmentation): U^n += nd s_d xi, U^(n-1) += nd s_d xi - nv s_v eta,
// xi, eta uniform in [-1, 1) from a hash of (cell, component, seed).
__device__ __forceinline__ float hash_uniform(unsigned a) {
    a ^= a >> 16; a *= 0x7feb352dU; a ^= a >> 15; a *= 0x846ca68bU; a ^= a >> 16;
    return (float)(a & 0xFFFFFFu) * (1.f / 8388608.f) - 1.f;
}
__global__ void k_noise(Mut4 now, Mut4 past, int pitch, Region rg, const unsigned* scale, float nd, float nv,
                        unsigned seed) {
    const int j = rg.r.j0 + blockIdx.x * blockDim.x + threadIdx.x, i = rg.r.i0 + blockIdx.y;
    if (j >= rg.r.j1 || !rg.in(i, j)) return;
    const float ad = __uint_as_float(scale[0]) * nd, av = __uint_as_float(scale[1]) * nv;
    const ptrdiff_t g = (ptrdiff_t)i * pitch + j;
    const unsigned base = seed * 0x9E3779B9u + (unsigned)(i * 8191 + j) * 16u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float a = hash_uniform(base + 2 * q) * ad, b = hash_uniform(base + 2 * q + 1) * av;
        now.f[q][g] += a;
        past.f[q][g] += a - b;
    }
}

// Fine state (pitch pf) restricted onto the coarse grid [Xc][Zc][4].
__global__ void k_restrict(Level4 fine, int pf, int Xc, int Zc, float* out) {
    const int jc = blockIdx.x * blockDim.x + threadIdx.x, ic = blockIdx.y;
    if (jc >= Zc) return;
    const int i = 2 * ic, j = 2 * jc;
    float* o = out + ((size_t)ic * Zc + jc) * 4;
#pragma unroll
    for (int q = 0; q < 4; q += 2) {   // x-staggered: Px, Sx
        const float* f = fine.f[q];
        o[q] = mid4(ld(f, pf, i - 1, j), ld(f, pf, i, j), ld(f, pf, i + 1, j), ld(f, pf, i + 2, j));
    }
#pragma unroll
    for (int q = 1; q < 4; q += 2) {   // z-staggered: Pz, Sz
        const float* f = fine.f[q];
        o[q] = mid4(ld(f, pf, i, j - 1), ld(f, pf, i, j), ld(f, pf, i, j + 1), ld(f, pf, i, j + 2));
    }
}

// Row rc of the coarse grid of the fine state: Ux, Uz at coarse cells (ic, rc).
__global__ void k_restrict_row(Level4 fine, int pf, int Xc, int rc, float* gx, float* gz) {
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if (ic >= Xc) return;
    const int i = 2 * ic, j = 2 * rc;
    float ux[4], uz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        ux[k] = ld(fine.f[0], pf, i - 1 + k, j) + ld(fine.f[2], pf, i - 1 + k, j);
        uz[k] = ld(fine.f[1], pf, i, j - 1 + k) + ld(fine.f[3], pf, i, j - 1 + k);
    }
    gx[ic] = mid4(ux[0], ux[1], ux[2], ux[3]);
    gz[ic] = mid4(uz[0], uz[1], uz[2], uz[3]);
}

// One pass of (1 4 6 4 1)/16 along x (axis 0) or z (axis 1) over [X][Z][C]
// images, zero outside the grid.
__global__ void k_binomial(const float* in, float* out, int X, int Z, int C, int axis) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= Z) return;
    const float w[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
    for (int c = 0; c < C; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int ii = axis == 0 ? i + k - 2 : i, jj = axis == 0 ? j : j + k - 2;
            if (ii >= 0 && ii < X && jj >= 0 && jj < Z) acc += w[k] * in[((size_t)ii * Z + jj) * C + c];
        }
        out[((size_t)i * Z + j) * C + c] = acc;
    }
}

// Zero an [X][Z][C] image outside the region.
__global__ void k_mask(float* a, int Z, int C, Region rg) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= Z || rg.in(i, j)) return;
    for (int c = 0; c < C; ++c) a[((size_t)i * Z + j) * C + c] = 0.f;
}

// Training target [X][Z][8] before the low-pass, zero outside the region; with d^n = truth^n - U^n
// and d^(n-1) likewise: G d^n / s_d, G (d^n - d^(n-1)) / s_v.
__global__ void k_target(const float* truth_cur, const float* truth_prev, Level4 now, Level4 past, int X, int Z,
                         int pitch, Region rg, const unsigned* scale, float* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= Z) return;
    float* o = out + ((size_t)i * Z + j) * kOut;
    const bool in = rg.in(i, j);
    const float id = kGain * inv_or_zero(scale[0]), iv = kGain * inv_or_zero(scale[1]);
    const ptrdiff_t g = (ptrdiff_t)i * pitch + j;
    const size_t c = ((size_t)i * Z + j) * 4;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float dn = truth_cur[c + q] - now.f[q][g], dp = truth_prev[c + q] - past.f[q][g];
        o[q] = in ? dn * id : 0.f;
        o[4 + q] = in ? (dn - dp) * iv : 0.f;
    }
}

// Restricted truth [X][Z][4] into the pitched state on the rectangle.
__global__ void k_set_state(const float* truth, int Z, int pitch, Rect r, Mut4 lvl) {
    const int j = r.j0 + blockIdx.x * blockDim.x + threadIdx.x, i = r.i0 + blockIdx.y;
    if (j >= r.j1) return;
    const float* t = truth + ((size_t)i * Z + j) * 4;
    const ptrdiff_t g = (ptrdiff_t)i * pitch + j;
#pragma unroll
    for (int q = 0; q < 4; ++q) lvl.f[q][g] = t[q];
}

Level4 view(float* const (&f)[4]) { return Level4{{f[0], f[1], f[2], f[3]}}; }
Mut4 mut(float* const (&f)[4]) { return Mut4{{f[0], f[1], f[2], f[3]}}; }
Rect interior(const ouc_ctx* c) { return Rect{c->L, c->X - c->L, c->L, c->Z - c->L}; }
// correction region of the shot whose descriptor was uploaded last (padded source cell)
Region region(const ouc_ctx* c, int sx, int sz) {
    return Region{Rect{c->L + kEdge, c->X - c->L - kEdge, c->L + kEdge, c->Z - c->L - kEdge}, sx, sz};
}

int ensure(ouc_ctx* c) {
    if (c->l_in) return OUC_OK;
    const size_t C = (size_t)c->X * c->Z;
    bool ok = cudaMalloc(&c->l_in, C * kIn * 4) == cudaSuccess && cudaMalloc(&c->l_out, C * kOut * 4) == cudaSuccess &&
              cudaMalloc(&c->l_truth, 2 * C * 4 * 4) == cudaSuccess && cudaMalloc(&c->l_scale, 2 * 4) == cudaSuccess &&
              cudaMalloc(&c->l_tmp, C * kOut * 4) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        cudaFree(c->l_in); cudaFree(c->l_out); cudaFree(c->l_truth); cudaFree(c->l_scale); cudaFree(c->l_tmp);
        c->l_in = c->l_out = c->l_truth = c->l_scale = c->l_tmp = nullptr;
        return host::fail(c, OUC_ENOMEM, "cannot allocate the corrector buffers");
    }
    c->bytes += C * (kIn + 2 * kOut + 8) * 4 + 8;
    return OUC_OK;
}

// Scales and network input of the state `s`.
void pack(ouc_ctx* c, const Side& s) {
    const Rect r = interior(c);
    unsigned* sc = reinterpret_cast<unsigned*>(c->l_scale);
    cudaMemsetAsync(sc, 0, 8, c->stream);
    k_scales<<<296, 256, 0, c->stream>>>(view(s.now), view(s.past), c->pitch, r, sc);
    k_pack_input<<<dim3((c->Z + 127) / 128, c->X), 128, 0, c->stream>>>(
        view(s.now), view(s.past), c->vp2, c->vs2, c->X, c->Z, c->pitch, c->cfg.dt / c->cfg.dx, sc, c->l_in);
    c->timing.kernel_launches += 2;
}

// S (x then z) of an [X][Z][8] image in place, then zero outside the region.
void lowpass(ouc_ctx* c, float* img, const Region& rg) {
    const dim3 g((c->Z + 127) / 128, c->X);
    k_binomial<<<g, 128, 0, c->stream>>>(img, c->l_tmp, c->X, c->Z, kOut, 0);
    k_binomial<<<g, 128, 0, c->stream>>>(c->l_tmp, img, c->X, c->Z, kOut, 1);
    k_mask<<<g, 128, 0, c->stream>>>(img, c->Z, kOut, rg);
    c->timing.kernel_launches += 3;
}

void apply(ouc_ctx* c, const Region& rg, Side& s) {
    lowpass(c, c->l_out, rg);
    k_apply<<<dim3((rg.r.j1 - rg.r.j0 + 127) / 128, rg.r.i1 - rg.r.i0), 128, 0, c->stream>>>(
        c->l_out, c->Z, c->pitch, rg, reinterpret_cast<unsigned*>(c->l_scale), mut(s.now), mut(s.past));
}

int correct(ouc_ctx* c, ouc_cnn* net, const Region& rg, Side& s) {
    pack(c, s);
    int rc = ouc_cnn_forward_dev(net, 1, c->X, c->Z, c->l_in, c->l_out, c->stream);
    if (rc) return host::fail(c, rc, "corrector forward failed");
    apply(c, rg, s);
    c->timing.kernel_launches += 5;
    return OUC_OK;
}

// The coarse context is the fine one at twice the spacing and time step.
int check_pair(ouc_ctx* fine, ouc_ctx* coarse) {
    auto near2 = [](float c, float f) { return std::fabs(c - 2.f * f) <= 1e-6f * std::fabs(c); };
    if (fine->X != 2 * coarse->X || fine->Z != 2 * coarse->Z || fine->L != 2 * coarse->L)
        return host::fail(coarse, OUC_EINVAL, "coarse grid must be the fine grid at half the cells (npml halved too)");
    if (!near2(coarse->cfg.dx, fine->cfg.dx) || !near2(coarse->cfg.dz, fine->cfg.dz) ||
        !near2(coarse->cfg.dt, fine->cfg.dt))
        return host::fail(coarse, OUC_EINVAL, "coarse spacing and time step must be twice the fine ones");
    if (fine->device != coarse->device) return host::fail(coarse, OUC_EINVAL, "contexts on different devices");
    return OUC_OK;
}

int check_even_shot(ouc_ctx* fine, const ouc_shot* s) {
    int rc = host::check_shot(fine, s);
    if (rc) return rc;
    if ((s->sx | s->sz | s->rz) & 1) return host::fail(fine, OUC_EINVAL, "fine source and receiver row must sit on even cells");
    return OUC_OK;
}

ouc_shot halve(const ouc_shot& s) {
    ouc_shot c = s;
    c.sx /= 2; c.sz /= 2; c.rz /= 2;
    return c;
}

}  // namespace learned
}  // namespace ouc

using namespace ouc;
using namespace ouc::learned;

extern "C" {

int ouc_coarse_wavelet(const float* fine, int nt_coarse, float* out) {
    if (!fine || !out || nt_coarse < 1) return OUC_EINVAL;
    for (int m = 0; m < nt_coarse; ++m) out[m] = 0.25f * fine[2 * m];
    return OUC_OK;
}

int ouc_forward_learned(ouc_ctx* ctx, ouc_cnn* net, const ouc_shot* shot, const float* wavelet, int every,
                        float* gather_vx, float* gather_vz) {
    if (!ctx) return OUC_EINVAL;
    int rc = host::check_shot(ctx, shot);
    if (rc) return rc;
    if (!wavelet) return host::fail(ctx, OUC_EINVAL, "wavelet is NULL");
    if (net && (every < 1 || every > ctx->nt)) return host::fail(ctx, OUC_EINVAL, "every must be in [1, nt]");
    cudaSetDevice(ctx->device);
    if (net && (rc = ensure(ctx))) return rc;
    ctx->step_phase = ouc_ctx::kIdle;
    ctx->timing = ouc_timing{};
    if (cudaMemcpyAsync(ctx->d_wavelet, wavelet, (size_t)ctx->nt * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return host::fail(ctx, OUC_ECUDA, "wavelet upload failed");
    if ((rc = host::upload_desc(ctx, 1, shot, ctx->d_wavelet))) return rc;
    if ((rc = host::zero_side(ctx, 1, 0, false))) return rc;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    Side s = ctx->src;
    StepArgs a = host::base_args(ctx);
    a.record = 1;
    const Region rg = region(ctx, shot->sx + ctx->L, shot->sz + ctx->L);
    for (int t = 0; t < ctx->nt; ++t) {
        if ((rc = host::fwd_step(ctx, a, s, 1, t))) return rc;
        if (net && (t + 1) % every == 0 && (rc = correct(ctx, net, rg, s))) return rc;
    }
    ctx->src = s;
    cudaEventRecord(ctx->ev[2], ctx->stream);
    if (gather_vx && (rc = host::gather_out(ctx, ctx->gather(0, 0), gather_vx, true))) return rc;
    if (gather_vz && (rc = host::gather_out(ctx, ctx->gather(0, 1), gather_vz, true))) return rc;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return host::cuda_fail(ctx, e, "learned forward");
    ctx->timing.forward_ms = host::elapsed(ctx->ev[1], ctx->ev[2]);
    if (net && ouc_cnn_error(net)) return host::fail(ctx, OUC_ETIMEOUT, "a corrector kernel wait ran out");
    return OUC_OK;
}

int ouc_forward_restricted(ouc_ctx* fine, const ouc_shot* shot, const float* wavelet, int nt_coarse,
                           float* gather_vx, float* gather_vz) {
    if (!fine) return OUC_EINVAL;
    int rc = check_even_shot(fine, shot);
    if (rc) return rc;
    if (!wavelet || !gather_vx || !gather_vz) return host::fail(fine, OUC_EINVAL, "NULL argument");
    if ((fine->X | fine->Z | fine->L) & 1) return host::fail(fine, OUC_EINVAL, "fine grid and npml must be even");
    if (nt_coarse < 1 || 2 * nt_coarse > fine->nt) return host::fail(fine, OUC_EINVAL, "nt_coarse must be in [1, nt/2]");
    cudaSetDevice(fine->device);
    fine->step_phase = ouc_ctx::kIdle;
    fine->timing = ouc_timing{};
    const int Xc = fine->X / 2, rc_row = (shot->rz + fine->L) / 2;
    if (cudaMemcpyAsync(fine->d_wavelet, wavelet, (size_t)fine->nt * 4, cudaMemcpyHostToDevice, fine->stream) != cudaSuccess)
        return host::fail(fine, OUC_ECUDA, "wavelet upload failed");
    if ((rc = host::upload_desc(fine, 1, shot, fine->d_wavelet))) return rc;
    if ((rc = host::zero_side(fine, 1, 0, false))) return rc;
    // time-major coarse gathers [nt_c][Xc] in the fine context's gather buffer
    float* gx = fine->gather(0, 0);
    float* gz = gx + (size_t)nt_coarse * Xc;
    Side s = fine->src;
    StepArgs a = host::base_args(fine);
    for (int t = 0; t < 2 * nt_coarse; ++t) {
        if ((rc = host::fwd_step(fine, a, s, 1, t))) return rc;
        if (t & 1) {   // level t + 1 = 2 (m + 1): coarse gather row m
            const int m = t / 2;
            k_restrict_row<<<(Xc + 127) / 128, 128, 0, fine->stream>>>(view(s.now), fine->pitch, Xc, rc_row,
                                                                         gx + (size_t)m * Xc, gz + (size_t)m * Xc);
            fine->timing.kernel_launches += 1;
        }
    }
    fine->src = s;
    const size_t n = (size_t)nt_coarse * Xc;
    std::vector<float> hx(n), hz(n);
    if (cudaMemcpyAsync(hx.data(), gx, n * 4, cudaMemcpyDeviceToHost, fine->stream) != cudaSuccess ||
        cudaMemcpyAsync(hz.data(), gz, n * 4, cudaMemcpyDeviceToHost, fine->stream) != cudaSuccess)
        return host::fail(fine, OUC_ECUDA, "gather download failed");
    const cudaError_t e = cudaStreamSynchronize(fine->stream);
    if (e != cudaSuccess) return host::cuda_fail(fine, e, "restricted forward");
    if (fine->cfg.gather_layout == OUC_GATHER_XT) {
        for (int m = 0; m < nt_coarse; ++m)
            for (int i = 0; i < Xc; ++i) {
                gather_vx[(size_t)i * nt_coarse + m] = hx[(size_t)m * Xc + i];
                gather_vz[(size_t)i * nt_coarse + m] = hz[(size_t)m * Xc + i];
            }
    } else {
        std::copy(hx.begin(), hx.end(), gather_vx);
        std::copy(hz.begin(), hz.end(), gather_vz);
    }
    return OUC_OK;
}

int ouc_learned_pairs(ouc_ctx* fine, ouc_ctx* coarse, ouc_cnn* net, const ouc_shot* shot, const float* wavelet,
                      int every, float noise, unsigned seed, int max_pairs, float* d_in, float* d_tgt, int* npairs) {
    if (!fine || !coarse || !npairs || !d_in || !d_tgt || !wavelet) return OUC_EINVAL;
    *npairs = 0;
    int rc = check_pair(fine, coarse);
    if (rc) return rc;
    if ((rc = check_even_shot(fine, shot))) return rc;
    if (every < 1 || 2 * every > fine->nt || every > coarse->nt) return host::fail(coarse, OUC_EINVAL, "bad every");
    cudaSetDevice(coarse->device);
    if ((rc = ensure(coarse))) return rc;
    fine->step_phase = coarse->step_phase = ouc_ctx::kIdle;
    const ouc_shot cshot = halve(*shot);
    std::vector<float> wc(coarse->nt, 0.f);
    const int ncw = std::min(coarse->nt, fine->nt / 2);
    ouc_coarse_wavelet(wavelet, ncw, wc.data());
    if (cudaMemcpyAsync(fine->d_wavelet, wavelet, (size_t)fine->nt * 4, cudaMemcpyHostToDevice, fine->stream) ||
        cudaMemcpyAsync(coarse->d_wavelet, wc.data(), (size_t)coarse->nt * 4, cudaMemcpyHostToDevice, coarse->stream))
        return host::fail(coarse, OUC_ECUDA, "wavelet upload failed");
    if ((rc = host::upload_desc(fine, 1, shot, fine->d_wavelet)) || (rc = host::upload_desc(coarse, 1, &cshot, coarse->d_wavelet)) ||
        (rc = host::zero_side(fine, 1, 0, false)) || (rc = host::zero_side(coarse, 1, 0, false)))
        return rc;
    // the fine stream's work must precede the coarse stream's use of it
    cudaEvent_t ev = fine->ev[3];
    const size_t C = (size_t)coarse->X * coarse->Z;
    float* t_cur = coarse->l_truth;
    float* t_prev = coarse->l_truth + C * 4;
    if (!(noise >= 0.f && noise < 1.f)) return host::fail(coarse, OUC_EINVAL, "noise must be in [0, 1)");
    const Rect r = interior(coarse);
    const Region rg = region(coarse, cshot.sx + coarse->L, cshot.sz + coarse->L);
    const dim3 gall((coarse->Z + 127) / 128, coarse->X), grect((r.j1 - r.j0 + 127) / 128, r.i1 - r.i0);
    const dim3 greg((rg.r.j1 - rg.r.j0 + 127) / 128, rg.r.i1 - rg.r.i0);
    Side sf = fine->src, sc = coarse->src;
    StepArgs af = host::base_args(fine), ac = host::base_args(coarse);
    int tf = 0, tc = 0, made = 0;
    const int last = std::min(coarse->nt, fine->nt / 2);
    for (int m = every; m <= last && made < max_pairs; m += every) {
        while (tf < 2 * m - 2)
            if ((rc = host::fwd_step(fine, af, sf, 1, tf++))) return rc;
        k_restrict<<<dim3((coarse->Z + 127) / 128, coarse->X), 128, 0, fine->stream>>>(view(sf.now), fine->pitch,
                                                                                      coarse->X, coarse->Z, t_prev);
        while (tf < 2 * m)
            if ((rc = host::fwd_step(fine, af, sf, 1, tf++))) return rc;
        k_restrict<<<dim3((coarse->Z + 127) / 128, coarse->X), 128, 0, fine->stream>>>(view(sf.now), fine->pitch,
                                                                                      coarse->X, coarse->Z, t_cur);
        cudaEventRecord(ev, fine->stream);
        while (tc < m)
            if ((rc = host::fwd_step(coarse, ac, sc, 1, tc++))) return rc;
        cudaStreamWaitEvent(coarse->stream, ev, 0);
        if (noise > 0.f) {   // augmentation: the network learns to remove perturbations it did not cause
            pack(coarse, sc);
            k_noise<<<greg, 128, 0, coarse->stream>>>(mut(sc.now), mut(sc.past), coarse->pitch, rg,
                                                      reinterpret_cast<unsigned*>(coarse->l_scale), noise, noise,
                                                      seed * 7919u + (unsigned)m);
        }
        pack(coarse, sc);
        unsigned sv = 0;
        cudaMemcpyAsync(&sv, coarse->l_scale + 1, 4, cudaMemcpyDeviceToHost, coarse->stream);
        if (cudaStreamSynchronize(coarse->stream) != cudaSuccess) return host::fail(coarse, OUC_ECUDA, "pair generation");
        if (sv != 0) {   // a pair with motion in it
            float* in = d_in + (size_t)made * C * kIn;
            float* tg = d_tgt + (size_t)made * C * kOut;
            cudaMemcpyAsync(in, coarse->l_in, C * kIn * 4, cudaMemcpyDeviceToDevice, coarse->stream);
            k_target<<<gall, 128, 0, coarse->stream>>>(t_cur, t_prev, view(sc.now), view(sc.past), coarse->X, coarse->Z,
                                                       coarse->pitch, rg, reinterpret_cast<unsigned*>(coarse->l_scale), tg);
            lowpass(coarse, tg, rg);
            ++made;
        }
        if (net) {
            // on-policy: the next interval starts from the corrected coarse state
            int e = ouc_cnn_forward_dev(net, 1, coarse->X, coarse->Z, coarse->l_in, coarse->l_out, coarse->stream);
            if (e) return host::fail(coarse, e, "corrector forward failed");
            apply(coarse, rg, sc);
        } else {
            // teacher forcing: the next interval starts from the fine solution
            k_set_state<<<grect, 128, 0, coarse->stream>>>(t_cur, coarse->Z, coarse->pitch, r, mut(sc.now));
            k_set_state<<<grect, 128, 0, coarse->stream>>>(t_prev, coarse->Z, coarse->pitch, r, mut(sc.past));
        }
        // the fine stream may overwrite the truth only after these reads
        cudaEventRecord(coarse->ev[3], coarse->stream);
        cudaStreamWaitEvent(fine->stream, coarse->ev[3], 0);
    }
    fine->src = sf;
    coarse->src = sc;
    const cudaError_t e = cudaStreamSynchronize(coarse->stream);
    if (e != cudaSuccess) return host::cuda_fail(coarse, e, "pair generation");
    if (cudaStreamSynchronize(fine->stream) != cudaSuccess) return host::fail(fine, OUC_ECUDA, "pair generation");
    *npairs = made;
    return OUC_OK;
}

}  // extern "C"
