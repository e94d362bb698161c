// Kernel instantiations and the small per-shot kernels (mute, imaging of
// the last level, image normalisation + Laplacian + FP64 stack, gather
// transposes, field packing).
#include <cuda_runtime.h>

#include <algorithm>

#include "fd_march.cuh"
#include "fd_step.cuh"
#include "ouc_internal.h"

namespace ouc {

template <int N, int MODE>
static cudaError_t configure_one() {
    cudaError_t e = cudaFuncSetAttribute(k_step<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, TileGeo<N>::bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_step<N, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_step_q<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, TileGeo<N>::bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_step_q<N, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_march<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, MarchGeo<N>::bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_march<N, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    return e;
}

template <int N>
static cudaError_t configure_modes() {
    cudaError_t e = configure_one<N, kFwd>();
    if (e == cudaSuccess) e = configure_one<N, kRcv>();
    if (e == cudaSuccess) e = configure_one<N, kRec>();
    return e;
}

// Shared-memory attributes of the step kernels of half-order N on the current
// device (a per-device setting): ouc_create sets them for its device, the
// no-allocation entry point at its set-up on each device.
cudaError_t configure_step_kernels(int N) {
    if (N == 2) return configure_modes<2>();
    if (N == 5) return configure_modes<5>();
    if (N == 6) return configure_modes<6>();
    return cudaErrorInvalidValue;
}

int march_segments(Mode mode, const StepArgs& a) {
    constexpr int RB = 16;
    const int row0 = mode == kRec ? (a.L / RB) * RB : 0;
    const int row_end = mode == kRec ? a.X - a.L : (a.X + RB - 1) / RB * RB;
    return (row_end - row0 + a.seg_rows - 1) / a.seg_rows;
}

template <int N, int MODE>
static void launch_one(const StepArgs& a, int tiles_x, int nshots, cudaStream_t s) {
    if (a.seg_rows > 0) {
        const int nseg = march_segments((Mode)MODE, a);
        k_march<N, MODE><<<dim3(nseg * a.tiles_z, nshots), kThreads, MarchGeo<N>::bytes, s>>>(a);
        return;
    }
    if (a.seg_rows < 0 && a.queue && a.order[MODE == kRec ? 1 : 0]) {
        const int ntiles = tiles_x * a.tiles_z;
        const int items = ntiles * nshots, grid = items < 2 * a.nsm ? items : 2 * a.nsm;
        k_step_q<N, MODE><<<grid, kThreads, TileGeo<N>::bytes, s>>>(a, nshots, ntiles);
        return;
    }
    constexpr int bytes = TileGeo<N>::bytes;
    k_step<N, MODE><<<dim3(tiles_x * a.tiles_z, nshots), kThreads, bytes, s>>>(a);
}

template <int N>
static int launch_mode(Mode m, const StepArgs& a, int tiles_x, int nshots, cudaStream_t s) {
    switch (m) {
        case kFwd: launch_one<N, kFwd>(a, tiles_x, nshots, s); return 0;
        case kRcv: launch_one<N, kRcv>(a, tiles_x, nshots, s); return 0;
        case kRec: launch_one<N, kRec>(a, tiles_x, nshots, s); return 0;
    }
    return 1;
}

// Refuses (returns 1) a launch whose state map is missing or whose now[]
// pointers are not fields of the mapped block, so that no step kernel runs
// a tensor copy with coordinates the map does not describe.
int launch_step(int N, Mode mode, const StepArgs& a, int tiles_x, int nshots, cudaStream_t s) {
    if (!a.state0 || a.fstride == 0 || a.nfields <= 0) return 1;
    StepArgs b = a;
    const float* f0 = a.state0 + (size_t)kGX * a.pitch + kZOFF;   // field 0 of slot 0, cell (0, 0)
    auto field_of = [&](const float* q) -> int {
        if (!q || q < f0) return -1;
        const size_t d = (size_t)(q - f0);
        return d % a.fstride == 0 && d / a.fstride < (size_t)a.nfields ? (int)(d / a.fstride) : -1;
    };
    for (int q = 0; q < 4; ++q) {
        b.now_field[q] = field_of(a.now[q]);
        if (b.now_field[q] < 0) return 1;
        b.past_field[q] = field_of(a.past[q]);
        b.rcv_field[q] = field_of(a.rcv[q]);
        if (q < 3) b.acc_field[q] = field_of(a.acc[q]);
        b.fold_field[q] = field_of(a.f_old[q]);
    }
    for (int q = 0; q < 8; ++q) b.o_field[q] = field_of(a.o[q]);
    switch (N) {
        case 2: return launch_mode<2>(mode, b, tiles_x, nshots, s);
        case 5: return launch_mode<5>(mode, b, tiles_x, nshots, s);
        case 6: return launch_mode<6>(mode, b, tiles_x, nshots, s);
    }
    return 1;
}

namespace {
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder() {
    static EncodeTiled fn = []() -> EncodeTiled {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

template <int N>
cudaError_t encode_for(StepArgs& a, const float* state0, int pitch, int rows, int nfields, int nslots, size_t fstride) {
    using G = TileGeo<N>;
    EncodeTiled enc = encoder();
    if (!enc) return cudaErrorNotSupported;
    // dimensions innermost first: columns, rows, fields, slots; strides in bytes
    const cuuint64_t dims[4] = {(cuuint64_t)pitch, (cuuint64_t)rows, (cuuint64_t)nfields, (cuuint64_t)nslots};
    const cuuint64_t strides[3] = {(cuuint64_t)pitch * 4, (cuuint64_t)fstride * 4, (cuuint64_t)fstride * nfields * 4};
    const cuuint32_t box[4] = {(cuuint32_t)G::UC, (cuuint32_t)G::UR, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    static_assert((G::UC * 4) % 16 == 0, "the box's rows are whole 16-byte units");
    if (reinterpret_cast<uintptr_t>(state0) % 16 != 0 || (pitch * 4) % 16 != 0 || (fstride * 4) % 16 != 0)
        return cudaErrorInvalidValue;
    const CUresult r = enc(&a.box_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(state0), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const cuuint32_t own[4] = {(cuuint32_t)G::TZ, (cuuint32_t)G::TX, 1, 1};
    const CUresult r2 = enc(&a.own_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(state0), dims, strides,
                            own, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r2 != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const cuuint32_t sbox[4] = {(cuuint32_t)G::SC, (cuuint32_t)G::SR, 1, 1};
    const CUresult r3 = enc(&a.s_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(state0), dims, strides,
                            sbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r3 != CUDA_SUCCESS) return cudaErrorInvalidValue;
    a.state0 = state0;
    a.fstride = fstride;
    a.nfields = nfields;
    return cudaSuccess;
}
}  // namespace

cudaError_t encode_box_map(StepArgs& a, const float* state0, int pitch, int rows, int nfields, int nslots,
                           size_t fstride, int N) {
    a.state0 = nullptr;
    if (N == 2) return encode_for<2>(a, state0, pitch, rows, nfields, nslots, fstride);
    if (N == 5) return encode_for<5>(a, state0, pitch, rows, nfields, nslots, fstride);
    if (N == 6) return encode_for<6>(a, state0, pitch, rows, nfields, nslots, fstride);
    return cudaErrorInvalidValue;
}

int step_smem_bytes(int N) {
    switch (N) {
        case 2: return TileGeo<2>::bytes;
        case 5: return TileGeo<5>::bytes;
        case 6: return TileGeo<6>::bytes;
    }
    return 0;
}

// Imaging at the last time level, where the reference correlates without a
// reconstruction step (corr_v at t = NT-1, PS:2361 after PS:2319-2324).
// Source P is the forward's final level; the receiver fields are the ones
// after the receiver's first back-step.
__global__ void k_image_only(const StepArgs p) {
    const int i = blockIdx.y + p.L;
    const size_t off = (size_t)blockIdx.z * p.shot_stride;
    for (int j = p.L + threadIdx.x + blockIdx.x * blockDim.x; j < p.Z - p.L; j += blockDim.x * gridDim.x) {
        const ptrdiff_t g = (ptrdiff_t)i * p.pitch + j + off;
        const float sx = p.now[0][g], sz = p.now[1][g];
        p.acc[0][g] += sx * p.rcv[0][g] + sz * p.rcv[1][g];
        p.acc[2][g] += sx * sx + sz * sz;
        p.acc[1][g] += sx * p.rcv[2][g] + sz * p.rcv[3][g];
    }
}

void launch_image_only(const StepArgs& a, int nshots, cudaStream_t s) {
    const int nx = a.X - 2 * a.L;
    dim3 grid((a.Z - 2 * a.L + 255) / 256, nx, nshots);
    k_image_only<<<grid, 256, 0, s>>>(a);
}

// image = num / illumination (image_fun, PS:1441-1455), then the 5-point
// Laplacian scaled by 1/dh^2 on [L+2, X-L-2) x [L+2, Z-L-2) (Laplace,
// PS:1457-1469), zero on the two-cell rim of the interior; written dense
// nx x nz and added into the FP64 stack.
__device__ __forceinline__ float img_at(const float* num, const float* den, ptrdiff_t g) { return num[g] / den[g]; }

// The same from compensated sums: value = acc - c, the quotient formed in
// double and rounded once.
__device__ __forceinline__ float img_at_comp(const float* num, const float* cn, const float* den, const float* cd,
                                             ptrdiff_t g) {
    return (float)(((double)num[g] - (double)cn[g]) / ((double)den[g] - (double)cd[g]));
}

__global__ void k_finalize(const FinalizeArgs f) {
    const int nx = f.X - 2 * f.L, nz = f.Z - 2 * f.L;
    const int ii = blockIdx.y;
    const int i = ii + f.L;
    for (int jj = threadIdx.x + blockIdx.x * blockDim.x; jj < nz; jj += blockDim.x * gridDim.x) {
        const int j = jj + f.L;
        const size_t o = (size_t)ii * nz + jj;
        double spp = 0.0, sps = 0.0, sil = 0.0;
        for (int b = 0; b < f.nshots; ++b) {   // shots in order: the FP64 stack is deterministic
            const ptrdiff_t g = (ptrdiff_t)i * f.pitch + j + (ptrdiff_t)(b * f.shot_stride);
            float lpp = 0.f, lps = 0.f;
            if (i >= f.L + 2 && i < f.X - f.L - 2 && j >= f.L + 2 && j < f.Z - f.L - 2) {
                const float* npp = f.acc[0];
                const float* nps = f.acc[1];
                const float* den = f.acc[2];
                const ptrdiff_t P = f.pitch;
                const float c = 1 / f.dh / f.dh;
                if (!f.comp[0]) {
                    lpp = c * (img_at(npp, den, g + P) + img_at(npp, den, g - P) - 2 * img_at(npp, den, g) +
                               img_at(npp, den, g + 1) + img_at(npp, den, g - 1) - 2 * img_at(npp, den, g));
                    lps = c * (img_at(nps, den, g + P) + img_at(nps, den, g - P) - 2 * img_at(nps, den, g) +
                               img_at(nps, den, g + 1) + img_at(nps, den, g - 1) - 2 * img_at(nps, den, g));
                } else {
                    const float *cpp = f.comp[0], *cps = f.comp[1], *cd = f.comp[2];
                    auto ip = [&](ptrdiff_t q) { return img_at_comp(npp, cpp, den, cd, q); };
                    auto is = [&](ptrdiff_t q) { return img_at_comp(nps, cps, den, cd, q); };
                    lpp = c * (ip(g + P) + ip(g - P) - 2 * ip(g) + ip(g + 1) + ip(g - 1) - 2 * ip(g));
                    lps = c * (is(g + P) + is(g - P) - 2 * is(g) + is(g + 1) + is(g - 1) - 2 * is(g));
                }
            }
            if (f.img) {
                f.img[((size_t)b * 2 + 0) * nx * nz + o] = lpp;
                f.img[((size_t)b * 2 + 1) * nx * nz + o] = lps;
            }
            spp += (double)lpp;
            sps += (double)lps;
            sil += f.illum_scale * (f.comp[2] ? (double)f.acc[2][g] - (double)f.comp[2][g] : (double)f.acc[2][g]);
        }
        if (f.stack[0] && !(f.status && *f.status)) {   // a failed batch leaves the stack as it was
            f.stack[0][o] += spp;
            f.stack[1][o] += sps;
            f.stack[2][o] += sil;
        }
    }
}

// Conversion of one f16 strip slot from the staging ring once its field
// maxima are complete (the forward step converts slot t-1 itself; this
// converts the last slot).  blockIdx.y = shot.
__global__ void k_strip_pack(const ShotDesc* shots, int slot, int ring, size_t strip_slot) {
    const ShotDesc& d = shots[blockIdx.y];
    const float* src = d.stage + (size_t)(slot & 1) * strip_slot;
    __half* dst = reinterpret_cast<__half*>(d.strips) + (size_t)slot * strip_slot;
    const unsigned* am = d.amax + (size_t)slot * kStripFields;
    for (size_t e = threadIdx.x + (size_t)blockIdx.x * blockDim.x; e < strip_slot; e += (size_t)blockDim.x * gridDim.x) {
        const int f = (int)(e / ring);
        dst[e] = __float2half_rn(scale2(src[e], f16_exp(am[f])));
    }
}

void launch_strip_pack(const ShotDesc* shots, int nshots, int slot, int ring, size_t strip_slot, cudaStream_t s) {
    const int blocks = (int)std::min<size_t>((strip_slot + 255) / 256, 1184);
    k_strip_pack<<<dim3(blocks, nshots), 256, 0, s>>>(shots, slot, ring, strip_slot);
}

// ---- source-wavefield snapshots ---------------------------------------------

__device__ __forceinline__ size_t snap_index(const SnapArgs& a, int b, int comp, int ii, int jj) {
    return (size_t)b * a.shot_elems + ((size_t)a.slot * 2 + comp) * a.nx * a.nz + (size_t)ii * a.nz + jj;
}

// Largest |Px|, |Pz| of each shot's interior (f16 snapshots): block maxima,
// then one atomic per block and component.  grid (z blocks, nx, shots).
__global__ void k_snap_amax(const SnapArgs a) {
    const int ii = blockIdx.y, b = blockIdx.z;
    const size_t off = (size_t)b * a.shot_stride;
    float m0 = 0.f, m1 = 0.f;
    for (int jj = threadIdx.x + blockIdx.x * blockDim.x; jj < a.nz; jj += blockDim.x * gridDim.x) {
        const ptrdiff_t g = (ptrdiff_t)(ii + a.L) * a.pitch + (jj + a.L) + off;
        m0 = fmaxf(m0, fabsf(a.px[g]));
        m1 = fmaxf(m1, fabsf(a.pz[g]));
    }
    __shared__ float red[2][32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m0 = fmaxf(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = fmaxf(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = m0; red[1][w] = m1; }
    __syncthreads();
    if (threadIdx.x < 2) {
        float m = 0.f;
        for (int q = 0; q < nw; ++q) m = fmaxf(m, red[threadIdx.x][q]);
        if (m > 0.f) atomicMax(a.amax + ((size_t)b * a.nslots + a.slot) * 2 + threadIdx.x, __float_as_uint(m));
    }
}

// Store the interior Px, Pz as snapshot `slot` in the snapshot type.
__global__ void k_snap_store(const SnapArgs a) {
    const int ii = blockIdx.y, b = blockIdx.z;
    const size_t off = (size_t)b * a.shot_stride;
    int k0 = 0, k1 = 0;
    if (a.prec == kStripF16) {
        const unsigned* am = a.amax + ((size_t)b * a.nslots + a.slot) * 2;
        k0 = f16_exp(am[0]);
        k1 = f16_exp(am[1]);
    }
    for (int jj = threadIdx.x + blockIdx.x * blockDim.x; jj < a.nz; jj += blockDim.x * gridDim.x) {
        const ptrdiff_t g = (ptrdiff_t)(ii + a.L) * a.pitch + (jj + a.L) + off;
        const float v0 = a.px[g], v1 = a.pz[g];
        const size_t e0 = snap_index(a, b, 0, ii, jj), e1 = snap_index(a, b, 1, ii, jj);
        if (a.prec == kStripF32) {
            static_cast<float*>(a.snaps)[e0] = v0;
            static_cast<float*>(a.snaps)[e1] = v1;
        } else if (a.prec == kStripBF16) {
            static_cast<__nv_bfloat16*>(a.snaps)[e0] = __float2bfloat16_rn(v0);
            static_cast<__nv_bfloat16*>(a.snaps)[e1] = __float2bfloat16_rn(v1);
        } else {
            static_cast<__half*>(a.snaps)[e0] = __float2half_rn(scale2(v0, k0));
            static_cast<__half*>(a.snaps)[e1] = __float2half_rn(scale2(v1, k1));
        }
    }
}

void launch_snap_store(const SnapArgs& a, int nshots, cudaStream_t s) {
    const dim3 grid((a.nz + 255) / 256, a.nx, nshots);
    if (a.prec == kStripF16) k_snap_amax<<<grid, 256, 0, s>>>(a);
    k_snap_store<<<grid, 256, 0, s>>>(a);
}

__device__ __forceinline__ float snap_get(const SnapArgs& a, size_t e, int k) {
    if (a.prec == kStripF32) return static_cast<const float*>(a.snaps)[e];
    if (a.prec == kStripBF16) return __bfloat162float(static_cast<const __nv_bfloat16*>(a.snaps)[e]);
    return scale2(__half2float(static_cast<const __half*>(a.snaps)[e]), -k);
}

__device__ __forceinline__ void kahan_add(float* acc, float* c, float term) {
    const float y = __fsub_rn(term, *c);
    const float t = __fadd_rn(*acc, y);
    *c = __fsub_rn(__fsub_rn(t, *acc), y);
    *acc = t;
}

// Zero-lag imaging at a snapshot level: the stored source P against the
// receiver wavefield after its back-step, with the rounding of corr_v
// (acc + fma(p, q, u v), PS:1434-1436).  grid (z blocks, nx, shots).
__global__ void k_image_snap(const SnapArgs a) {
    const int ii = blockIdx.y, b = blockIdx.z;
    const size_t off = (size_t)b * a.shot_stride;
    int k0 = 0, k1 = 0;
    if (a.prec == kStripF16) {
        const unsigned* am = a.amax + ((size_t)b * a.nslots + a.slot) * 2;
        k0 = f16_exp(am[0]);
        k1 = f16_exp(am[1]);
    }
    for (int jj = threadIdx.x + blockIdx.x * blockDim.x; jj < a.nz; jj += blockDim.x * gridDim.x) {
        const ptrdiff_t g = (ptrdiff_t)(ii + a.L) * a.pitch + (jj + a.L) + off;
        const float sx = snap_get(a, snap_index(a, b, 0, ii, jj), k0);
        const float sz = snap_get(a, snap_index(a, b, 1, ii, jj), k1);
        const float rpx = a.rcv[0][g], rpz = a.rcv[1][g], rsx = a.rcv[2][g], rsz = a.rcv[3][g];
        const float tpp = __fmaf_rn(sx, rpx, __fmul_rn(sz, rpz));
        const float tps = __fmaf_rn(sx, rsx, __fmul_rn(sz, rsz));
        const float til = __fmaf_rn(sx, sx, __fmul_rn(sz, sz));
        if (!a.comp_image) {
            a.acc[0][g] = __fadd_rn(a.acc[0][g], tpp);
            a.acc[1][g] = __fadd_rn(a.acc[1][g], tps);
            a.acc[2][g] = __fadd_rn(a.acc[2][g], til);
        } else {
            kahan_add(a.acc[0] + g, a.comp[0] + g, tpp);
            kahan_add(a.acc[1] + g, a.comp[1] + g, tps);
            kahan_add(a.acc[2] + g, a.comp[2] + g, til);
        }
    }
}

void launch_image_snap(const SnapArgs& a, int nshots, cudaStream_t s) {
    k_image_snap<<<dim3((a.nz + 255) / 256, a.nx, nshots), 256, 0, s>>>(a);
}

void launch_finalize(const FinalizeArgs& f, cudaStream_t s) {
    const int nx = f.X - 2 * f.L, nz = f.Z - 2 * f.L;
    dim3 grid((nz + 255) / 256, nx);
    k_finalize<<<grid, 256, 0, s>>>(f);
}

// Direct-wave mute (remove, PS:1634-1657) on a time-major gather [nt][X]:
// zero sample t of receiver i when t < 2 t0 + dist(i) * dh / (dt * v), with
// the reference's mix of float and double arithmetic.
__global__ void k_mute(float* gx, float* gz, int X, int nt, int sx, int sz, int rz, int t0, float dt, float dh,
                       float v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= X) return;
    const int dxi = abs(sx - i), dzi = abs(rz - sz);
    const float dist = sqrtf(float(dxi * dxi + dzi * dzi));
    const double thr = 2 * t0 + (double)(dist * dh) * 1.0 / (double)(dt * v);
    for (int t = blockIdx.y; t < nt; t += gridDim.y) {
        if (t < thr) {
            gx[(size_t)t * X + i] = 0.f;
            gz[(size_t)t * X + i] = 0.f;
        }
    }
}

void launch_mute(float* gx, float* gz, int X, int nt, int sx, int sz, int rz, int t0, float dt, float dh, float v,
                 cudaStream_t s) {
    dim3 grid((X + 127) / 128, nt < 1024 ? nt : 1024);
    k_mute<<<grid, 128, 0, s>>>(gx, gz, X, nt, sx, sz, rz, t0, dt, dh, v);
}

// Non-finite detector: bit 1 of *status when any of the n floats at p is
// NaN or infinite (an unstable or overflowing run).  One vote per warp, one
// atomic per warp that saw one; the data is only read.
__global__ void k_finite(const float* __restrict__ p, size_t n, int* status) {
    bool bad = false;
    const size_t n4 = n / 4;
    const float4* p4 = reinterpret_cast<const float4*>(p);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
        const float4 v = p4[i];
        bad |= !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w);
    }
    for (size_t i = 4 * n4 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        bad |= !isfinite(p[i]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, 2);
}

void launch_finite_check(const float* p, size_t n, int* status, cudaStream_t s) {
    k_finite<<<1184, 256, 0, s>>>(p, n, status);   // 8 CTAs of 256 per SM, grid-stride
}

// out[c][r] = in[r][c] through a 32x33 shared tile.
__global__ void k_transpose(const float* __restrict__ in, float* __restrict__ out, int rows, int cols) {
    __shared__ float tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][k];
    }
}

void launch_transpose(const float* in, float* out, int rows, int cols, cudaStream_t s) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    k_transpose<<<grid, dim3(32, 8), 0, s>>>(in, out, rows, cols);
}

// Gather nf pitched fields into a dense [nf][X][Z] buffer.
// FWI gradient of one back-step (the formula of the reference's unused
// gradfun, PS:1518-1575), for every shot of the launch (blockIdx.y):
//   G_vp -= 2 rho Vp (dUx/dx + dUz/dz) theta_r
//   G_vs -= 2 rho Vs (omega_r (dUx/dz - dUz/dx) + Qzx_r dUz/dx + Qzz_r dUz/dz + Qxz_r dUx/dz + Qxx_r dUx/dx)
//   S    += Ux_s^2 + Uz_s^2
// with U_s = P + S of the source at the imaged level, its staggered
// derivatives (dUx/dx = D-x, dUz/dz = D-z, dUz/dx = D+x, dUx/dz = D+z), and
// the receiver's stress fields from U_r = P + S after the back-step
// (PS:373-378 without damping memories), on [L+N, X-L-N) x [L+N, Z-L-N):
// every stencil reads interior cells only.  A CTA stages the four U fields
// of a 16 x 64 tile with an N-row and 8-column halo in shared memory.
template <int N>
__global__ void __launch_bounds__(256) k_grad(const GradArgs a) {
    constexpr int TR = 16, TC = 64, HC = 8, BR = TR + 2 * N, BC = TC + 2 * HC;
    __shared__ float4 sbox4[4 * BR * BC / 4];
    float* box = reinterpret_cast<float*>(sbox4);
    const int b = blockIdx.y;
    const int tiles_c = (a.Z + TC - 1) / TC;
    const int x0 = (blockIdx.x / tiles_c) * TR, z0 = (blockIdx.x % tiles_c) * TC;
    const size_t off = (size_t)b * a.shot_stride;
    for (int k = threadIdx.x; k < BR * (BC / 4); k += blockDim.x) {
        const int r = k / (BC / 4), c4 = k - r * (BC / 4);
        const ptrdiff_t g = (ptrdiff_t)(x0 - N + r) * a.pitch + (z0 - HC + 4 * c4);
        const float4 spx = *reinterpret_cast<const float4*>(a.src[0] + off + g);
        const float4 spz = *reinterpret_cast<const float4*>(a.src[1] + off + g);
        const float4 ssx = *reinterpret_cast<const float4*>(a.src[2] + off + g);
        const float4 ssz = *reinterpret_cast<const float4*>(a.src[3] + off + g);
        const float4 rpx = *reinterpret_cast<const float4*>(a.rcv[0] + off + g);
        const float4 rpz = *reinterpret_cast<const float4*>(a.rcv[1] + off + g);
        const float4 rsx = *reinterpret_cast<const float4*>(a.rcv[2] + off + g);
        const float4 rsz = *reinterpret_cast<const float4*>(a.rcv[3] + off + g);
        float4* o = sbox4 + r * (BC / 4) + c4;
        o[0 * BR * BC / 4] = make_float4(spx.x + ssx.x, spx.y + ssx.y, spx.z + ssx.z, spx.w + ssx.w);
        o[1 * BR * BC / 4] = make_float4(spz.x + ssz.x, spz.y + ssz.y, spz.z + ssz.z, spz.w + ssz.w);
        o[2 * BR * BC / 4] = make_float4(rpx.x + rsx.x, rpx.y + rsx.y, rpx.z + rsx.z, rpx.w + rsx.w);
        o[3 * BR * BC / 4] = make_float4(rpz.x + rsz.x, rpz.y + rsz.y, rpz.z + rsz.z, rpz.w + rsz.w);
    }
    __syncthreads();
    const float* usx = box;
    const float* usz = box + BR * BC;
    const float* urx = box + 2 * BR * BC;
    const float* urz = box + 3 * BR * BC;
    auto at = [&](const float* f, int r, int c) { return f[(r + N) * BC + (c + HC)]; };
    // staggered derivatives at tile cell (r, c), PS:224-279 stencil forms
    auto dmx = [&](const float* f, int r, int c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 1; k <= N; ++k) acc = fmaf(a.a[k - 1], at(f, r + k - 1, c) - at(f, r - k, c), acc);
        return acc / a.dx;
    };
    auto dpx = [&](const float* f, int r, int c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 1; k <= N; ++k) acc = fmaf(a.a[k - 1], at(f, r + k, c) - at(f, r - k + 1, c), acc);
        return acc / a.dx;
    };
    auto dmz = [&](const float* f, int r, int c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 1; k <= N; ++k) acc = fmaf(a.a[k - 1], at(f, r, c + k - 1) - at(f, r, c - k), acc);
        return acc / a.dz;
    };
    auto dpz = [&](const float* f, int r, int c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 1; k <= N; ++k) acc = fmaf(a.a[k - 1], at(f, r, c + k) - at(f, r, c - k + 1), acc);
        return acc / a.dz;
    };
    const int r = threadIdx.x / (TC / 4), c0 = 4 * (threadIdx.x % (TC / 4));
    const int i = x0 + r;
    if (r >= TR || i < a.L + N || i >= a.X - a.L - N) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int c = c0 + q, j = z0 + c;
        if (j < a.L + N || j >= a.Z - a.L - N) continue;
        const float sxx = dmx(usx, r, c), szz = dmz(usz, r, c), szx = dpx(usz, r, c), sxz = dpz(usx, r, c);
        const float rxx = dmx(urx, r, c), rzz = dmz(urz, r, c), rzx = dpx(urz, r, c), rxz = dpz(urx, r, c);
        const ptrdiff_t g = (ptrdiff_t)i * a.pitch + j;
        const float vp = a.vp[g], vs = a.vs[g], vp2 = vp * vp, vs2 = vs * vs;
        const float rho = a.rho ? a.rho[g] : 1.f;
        const float th = vp2 * (rxx + rzz), om = vs2 * (rxz - rzx);
        const float s_vs = om * (sxz - szx) + vs2 * rzx * szx + vs2 * rzz * szz + vs2 * rxz * sxz + vs2 * rxx * sxx;
        const size_t og = (size_t)b * a.grad_stride + g;
        a.g[0][og] -= 2.f * rho * vp * ((sxx + szz) * th);
        a.g[1][og] -= 2.f * rho * vs * s_vs;
        const float ux = at(usx, r, c), uz = at(usz, r, c);
        a.g[2][og] += ux * ux + uz * uz;
    }
}

void launch_grad(const GradArgs& a, cudaStream_t s) {
    // tile rows only up to the last gradient row X-L-N-1: the staged rows then
    // end below X-L+14, inside the fields' 16 guard rows
    const int tiles = ((a.X - a.L - a.N + 15) / 16) * ((a.Z + 63) / 64);
    const dim3 grid(tiles, a.nshots);
    if (a.N == 2) k_grad<2><<<grid, 256, 0, s>>>(a);
    else if (a.N == 5) k_grad<5><<<grid, 256, 0, s>>>(a);
    else k_grad<6><<<grid, 256, 0, s>>>(a);
}

// FP64 stack of the shots' gradients over the interior, shots in order.
__global__ void k_grad_stack(const GradStackArgs a) {
    const int nz = a.Z - 2 * a.L;
    const int ii = blockIdx.y, i = ii + a.L;
    for (int jj = threadIdx.x + blockIdx.x * blockDim.x; jj < nz; jj += blockDim.x * gridDim.x) {
        const ptrdiff_t g = (ptrdiff_t)i * a.pitch + jj + a.L;
        double s[3] = {0.0, 0.0, 0.0};
        for (int b = 0; b < a.nshots; ++b)
            for (int k = 0; k < 3; ++k) s[k] += (double)a.g[k][(size_t)b * a.grad_stride + g];
        for (int k = 0; k < 3; ++k) a.stack[k][(size_t)ii * nz + jj] += s[k];
    }
}

void launch_grad_stack(const GradStackArgs& a, cudaStream_t s) {
    const int nz = a.Z - 2 * a.L, nx = a.X - 2 * a.L;
    k_grad_stack<<<dim3((nz + 255) / 256, nx), 256, 0, s>>>(a);
}

struct PackArgs {
    const float* f[12];
    int nf, X, Z, pitch;
    float* out;
};
__global__ void k_pack(const PackArgs a) {
    const int i = blockIdx.y, k = blockIdx.z;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < a.Z; j += blockDim.x * gridDim.x)
        a.out[((size_t)k * a.X + i) * a.Z + j] = a.f[k][(ptrdiff_t)i * a.pitch + j];
}

void launch_pack_fields(const float* const* f, int nf, int X, int Z, int pitch, float* out, cudaStream_t s) {
    PackArgs a;
    for (int k = 0; k < nf && k < 12; ++k) a.f[k] = f[k];
    a.nf = nf; a.X = X; a.Z = Z; a.pitch = pitch; a.out = out;
    dim3 grid((Z + 255) / 256, X, nf);
    k_pack<<<grid, 256, 0, s>>>(a);
}

}  // namespace ouc
