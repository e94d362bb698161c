// Forward modeling without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// forward-modeling run: host applications that hand the whole GPU to a
// memory pool of their own and forbid any other allocation, and pipelines
// that reserve all device memory up front and must not call the allocator
// later (cudaMalloc and cudaFree synchronise the device and can fail under
// memory pressure).  ouc_forward_noalloc serves them: it runs the same
// forward-step kernels as ouc_forward, but its wavefield state, model fields
// and gather staging live in one fixed array, g_scratch below, that is part
// of the library image.  The caller passes only its own inputs (padded
// model, wavelet) and outputs (gathers) as device pointers.
//
// Properties a caller must know:
//   * g_scratch is OUC_NOALLOC_SCRATCH_BYTES (64 MiB) of device memory on
//     every GPU that loads this part of the library (with CUDA's default lazy
//     module loading, from the first call on that GPU), held until the
//     process exits;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and sets the step kernels' shared-memory limit
//     on that device -- make that first call before any stream capture on
//     that device;
//   * all calls share the one array and it keeps the previous call's
//     contents: every call clears what must start at zero, and calls whose
//     work overlaps on the GPU (different streams, or different host
//     threads) race on it -- serialise them;
//   * problems that do not fit the array are rejected with OUC_ESCRATCH;
//   * the step kernels' copy waits are bounded; the call itself returns
//     before they run, so a wait that gives up (no such case is known) is
//     reported in the output: both gathers are filled with NaN.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/ouc.h"
#include "ouc_internal.h"

using namespace ouc;

namespace {

constexpr size_t kScratchFloats = OUC_NOALLOC_SCRATCH_BYTES / sizeof(float);
constexpr int kMaxDevices = 64;
constexpr int kMaxPml = 255;

__device__ __align__(256) float g_scratch[kScratchFloats];

// Device address of g_scratch per device ordinal (host-side cache).
float* g_scratch_addr[kMaxDevices] = {};

struct ModelArgs {
    const float* vp;         // caller's padded model, dense X x Z
    const float* vs;
    float* vp2;              // pitched outputs
    float* vs2;
    float* ax;
    float* az;
    int X, Z, L, pitch;
    double c;                // log10(1/R) * 1.5
    double pw[kMaxPml + 1];  // pow(k / L, 4) for k = 0..L, computed on the host
};

// Model fields in the pitched layout: Vp^2, Vs^2 and the damping profile of
// PS:2067-2105, evaluated as (c * v) / L * pw[k] in double exactly as the
// host set-up of ouc_create does, so both entry points see the same floats.
__global__ void k_model(const ModelArgs m) {
    const int i = blockIdx.y;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < m.Z; j += blockDim.x * gridDim.x) {
        const float v = m.vp[(size_t)i * m.Z + j], s = m.vs[(size_t)i * m.Z + j];
        const ptrdiff_t g = (ptrdiff_t)i * m.pitch + j;
        m.vp2[g] = v * v;
        m.vs2[g] = s * s;
        const double dv = v;
        float ax = 0.f, az = 0.f;
        if (i < m.L) ax = (float)(m.c * dv / m.L * m.pw[m.L - i]);
        else if (i > m.X - m.L) ax = (float)(m.c * dv / m.L * m.pw[i - m.X + m.L]);
        if (j < m.L) az = (float)(m.c * dv / m.L * m.pw[m.L - j]);
        else if (j > m.Z - m.L) az = (float)(m.c * dv / m.L * m.pw[j - m.Z + m.L]);
        m.ax[g] = ax;
        m.az[g] = az;
    }
}

// The shot descriptor is written by the device from a by-value kernel
// argument, so the call queues only kernels, memsets and device-to-device
// copies (no host-to-device copy from pageable memory).
__global__ void k_put_desc(ShotDesc* dst, const ShotDesc desc) { *dst = desc; }

// After the run: if a step kernel recorded a failed copy wait, mark the
// caller's gathers as invalid (NaN) -- the only report an asynchronous call
// can give.
__global__ void k_mark_failed(const int* status, float* gx, float* gz, size_t n) {
    if (!(*status & 1)) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        gx[i] = __int_as_float(0x7fc00000);
        gz[i] = __int_as_float(0x7fc00000);
    }
}

}  // namespace

extern "C" int ouc_forward_noalloc(const ouc_config* cfg, const ouc_shot* shot, const float* d_vp,
                                   const float* d_vs, const float* d_wavelet, float* d_gather_vx,
                                   float* d_gather_vz) {
    if (!cfg || !shot || !d_vp || !d_vs || !d_wavelet || !d_gather_vx || !d_gather_vz) return OUC_EINVAL;
    const int N = cfg->half_order, L = cfg->npml;
    if (N != 2 && N != 5 && N != 6) return OUC_EINVAL;
    // this entry point reads a padded X x Z model, runs the density-normalised
    // equations and writes one of the two gather layouts; anything else is
    // refused before any device work
    if (cfg->model_layout != OUC_MODEL_PADDED || cfg->density != 0) return OUC_EINVAL;
    if (cfg->gather_layout != OUC_GATHER_XT && cfg->gather_layout != OUC_GATHER_TX) return OUC_EINVAL;
    if (cfg->nx < 4 * N || cfg->nz < 4 * N || L < N || L > kMaxPml || cfg->nt < 2) return OUC_EINVAL;
    // sizes in 64-bit before any derived extent: X, Z and the pitch stay far
    // below INT_MAX for every grid that can fit the array
    if ((long long)cfg->nx + 2LL * L > (1LL << 24) || (long long)cfg->nz + 2LL * L > (1LL << 24) ||
        (long long)cfg->nt > (1LL << 30))
        return OUC_ESCRATCH;
    if (!(cfg->dx > 0) || !(cfg->dz > 0) || !(cfg->dt > 0) || cfg->dx > 256.f || cfg->dz > 256.f) return OUC_EINVAL;
    if (!(cfg->pml_r > 0 && cfg->pml_r < 1)) return OUC_EINVAL;
    if (shot->sx < 0 || shot->sx >= cfg->nx || shot->sz < 0 || shot->sz >= cfg->nz || shot->rz < 0 ||
        shot->rz >= cfg->nz || (shot->src_type != OUC_SRC_THETA && shot->src_type != OUC_SRC_FORCE_Z))
        return OUC_EINVAL;
    cudaStream_t stream = (cudaStream_t)cfg->stream;
    // an error left by the caller's own earlier work is theirs to read: report
    // it without clearing it, before queueing anything
    if (cudaPeekAtLastError() != cudaSuccess) return OUC_ECUDA;

    // set-up, once per device: the array's device address
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return OUC_ENODEV;
    if (!g_scratch_addr[dev]) {
        float* ptr = nullptr;
        if (cudaGetSymbolAddress((void**)&ptr, g_scratch) != cudaSuccess || !ptr) return OUC_ECUDA;
        // the step kernels' shared-memory opt-in is a per-device setting too
        for (int n : {2, 5, 6})
            if (configure_step_kernels(n) != cudaSuccess) {
                cudaGetLastError();   // this call's own failure: clear it, report it
                return OUC_ECUDA;
            }
        g_scratch_addr[dev] = ptr;
    }
    float* base = g_scratch_addr[dev];

    // layout: the same pitched padded grid as ouc_create
    const int X = cfg->nx + 2 * L, Z = cfg->nz + 2 * L, nt = cfg->nt;
    const TileGrid tg = tile_grid(X, Z, L);
    const int tiles_x = tg.tiles_x, tiles_z = tg.tiles_z;
    const int Xc = tg.Xc, Zc = tg.Zc;
    const int pitch = ((kZOFF + Zc + kZOFF) + 31) / 32 * 32;
    const size_t fstride = (size_t)(Xc + 2 * kGX) * pitch;
    const size_t nfields = 4 + 24;   // model: vp2 vs2 ax az; state: now 4, past 4, F 2x4, O 8
    const size_t gather_floats = 2 * (size_t)nt * X;
    const size_t desc_at = (nfields * fstride + gather_floats + 63) / 64 * 64;   // 256-byte aligned
    const size_t status_at = desc_at + (sizeof(ShotDesc) + 3) / 4;   // one int: the kernels' status word
    const size_t need = status_at + 1;
    if (need > kScratchFloats) return OUC_ESCRATCH;
    auto field = [&](size_t k) { return base + k * fstride + (size_t)kGX * pitch + kZOFF; };
    float* gathers = base + nfields * fstride;
    ShotDesc* d_desc = reinterpret_cast<ShotDesc*>(base + desc_at);
    int* d_status = reinterpret_cast<int*>(base + status_at);

    // clear everything this call reads before writing (previous calls' contents)
    if (cudaMemsetAsync(base, 0, nfields * fstride * sizeof(float), stream) != cudaSuccess) return OUC_ECUDA;
    if (cudaMemsetAsync(d_status, 0, sizeof(int), stream) != cudaSuccess) return OUC_ECUDA;

    ModelArgs m;
    memset(&m, 0, sizeof(m));
    m.vp = d_vp; m.vs = d_vs;
    m.vp2 = field(0); m.vs2 = field(1); m.ax = field(2); m.az = field(3);
    m.X = X; m.Z = Z; m.L = L; m.pitch = pitch;
    m.c = log10(1.0 / cfg->pml_r) * 1.5;
    for (int k = 0; k <= L; ++k) m.pw[k] = pow(1.0 * k / L, 4.0);
    k_model<<<dim3((Z + 255) / 256, X), 256, 0, stream>>>(m);

    ShotDesc desc;
    memset(&desc, 0, sizeof(desc));
    desc.sx = shot->sx + L; desc.sz = shot->sz + L; desc.rz = shot->rz + L;
    desc.src_type = shot->src_type;
    desc.wavelet = d_wavelet;
    desc.gather_x = gathers;
    desc.gather_z = gathers + (size_t)nt * X;
    desc.strips = nullptr;
    desc.X = X;
    desc.tiles_x = tiles_x;
    desc.rec_tiles_x = tiles_x;
    desc.ring = Ring::make(X, Z, L, N);
    desc.off = 0;
    desc.strip_slot = 0;
    desc.vp2 = field(0); desc.vs2 = field(1); desc.ax = field(2); desc.az = field(3);
    desc.bx = nullptr; desc.bz = nullptr;   // density-normalised equations only
    k_put_desc<<<1, 1, 0, stream>>>(d_desc, desc);

    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.X = X; a.Z = Z; a.pitch = pitch; a.L = L;
    a.tiles_z = tiles_z;
    for (int k = 0; k < N; ++k) a.a[k] = (float)kStencilWeights[N][k];
    a.dx = cfg->dx; a.dz = cfg->dz; a.dt = cfg->dt; a.dt2 = cfg->dt * cfg->dt;
    a.rdx = 1.0f / cfg->dx; a.rdz = 1.0f / cfg->dz;
    a.vp2 = field(0); a.vs2 = field(1); a.ax = field(2); a.az = field(3);
    a.shot_stride = 0;
    a.ring = Ring::make(X, Z, L, N);
    a.shots = d_desc;
    a.err = d_status;
    a.record = 1;
    // the tensor map of the scratch state block (its four leapfrog fields
    // start at field 4); encoded on the host, passed with the arguments
    if (encode_box_map(a, base, pitch, Xc + 2 * kGX, (int)nfields, 1, fstride, N) != cudaSuccess) return OUC_ECUDA;
    a.save = 0;
    float *now[4], *past[4], *fo[4], *fn[4], *o[8];
    size_t k = 4;
    for (int q = 0; q < 4; ++q) now[q] = field(k++);
    for (int q = 0; q < 4; ++q) past[q] = field(k++);
    for (int q = 0; q < 4; ++q) fo[q] = field(k++);
    for (int q = 0; q < 4; ++q) fn[q] = field(k++);
    for (int q = 0; q < 8; ++q) o[q] = field(k++);
    for (int t = 0; t < nt; ++t) {
        for (int q = 0; q < 4; ++q) {
            a.now[q] = now[q]; a.past[q] = past[q]; a.f_old[q] = fo[q]; a.f_new[q] = fn[q];
        }
        for (int q = 0; q < 8; ++q) a.o[q] = o[q];
        a.t = t;
        if (launch_step(N, kFwd, a, tiles_x, 1, stream)) return OUC_EINVAL;
        for (int q = 0; q < 4; ++q) {
            float* tmp = now[q]; now[q] = past[q]; past[q] = tmp;
            tmp = fo[q]; fo[q] = fn[q]; fn[q] = tmp;
        }
    }
    // time-major staging -> the caller's layout
    if (cfg->gather_layout == OUC_GATHER_XT) {
        launch_transpose(gathers, d_gather_vx, nt, X, stream);
        launch_transpose(gathers + (size_t)nt * X, d_gather_vz, nt, X, stream);
    } else {
        if (cudaMemcpyAsync(d_gather_vx, gathers, (size_t)nt * X * 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
            cudaMemcpyAsync(d_gather_vz, gathers + (size_t)nt * X, (size_t)nt * X * 4, cudaMemcpyDeviceToDevice,
                            stream) != cudaSuccess)
            return OUC_ECUDA;
    }
    k_mark_failed<<<148, 256, 0, stream>>>(d_status, d_gather_vx, d_gather_vz, (size_t)nt * X);
    return cudaGetLastError() == cudaSuccess ? OUC_OK : OUC_ECUDA;
}
