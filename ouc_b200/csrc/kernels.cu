// Kernel instantiations and the small per-shot kernels (mute, imaging of
// the last level, image normalisation + Laplacian + FP64 stack, gather
// transposes, field packing).
#include <cuda_runtime.h>

#include "fd_step.cuh"
#include "ouc_internal.h"

namespace ouc {

template <int N, int MODE>
static void launch_one(const StepArgs& a, int tiles_x, int nshots, cudaStream_t s) {
    constexpr int bytes = TileGeo<N>::bytes;
    static bool configured = false;   // one attribute call per instantiation
    if (!configured) {
        cudaFuncSetAttribute(k_step<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(k_step<N, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        configured = true;
    }
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

int launch_step(int N, Mode mode, const StepArgs& a, int tiles_x, int nshots, cudaStream_t s) {
    switch (N) {
        case 2: return launch_mode<2>(mode, a, tiles_x, nshots, s);
        case 5: return launch_mode<5>(mode, a, tiles_x, nshots, s);
        case 6: return launch_mode<6>(mode, a, tiles_x, nshots, s);
    }
    return 1;
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
                lpp = c * (img_at(npp, den, g + P) + img_at(npp, den, g - P) - 2 * img_at(npp, den, g) +
                           img_at(npp, den, g + 1) + img_at(npp, den, g - 1) - 2 * img_at(npp, den, g));
                lps = c * (img_at(nps, den, g + P) + img_at(nps, den, g - P) - 2 * img_at(nps, den, g) +
                           img_at(nps, den, g + 1) + img_at(nps, den, g - 1) - 2 * img_at(nps, den, g));
            }
            if (f.img) {
                f.img[((size_t)b * 2 + 0) * nx * nz + o] = lpp;
                f.img[((size_t)b * 2 + 1) * nx * nz + o] = lps;
            }
            spp += (double)lpp;
            sps += (double)lps;
            sil += (double)f.acc[2][g];
        }
        if (f.stack[0]) {
            f.stack[0][o] += spp;
            f.stack[1][o] += sps;
            f.stack[2][o] += sil;
        }
    }
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
