// Learned dispersion corrector (include/ouc_corrector.h): a 4-layer 5x5 CNN
// whose convolutions run as implicit GEMMs on the sm_100a tensor cores.
//
// One convolution tile = 128 consecutive pixels of one image row (GEMM M),
// all output channels (N = 32 or 16), K = 25 taps x input channels.  The CTA
// stages the 5-row x 132-column input patch in shared memory in the
// no-swizzle K-major "core matrix" layout -- [row][channel chunk of 8][column]
// [8 channels], 16 bytes per (column, chunk) -- so that the A operand of tap
// (dx, dz) is simply the patch shifted by (dx, dz): a shared-memory matrix
// descriptor whose start address moves by 16 * (dx * chunks * 132 + dz)
// bytes, with the leading-dimension offset = one chunk plane (132 * 16 B)
// and the stride offset = 8 pixels (128 B).  No im2col copy is made.  The
// weights of all taps sit in shared memory for the whole (persistent) CTA in
// the same layout, [tap][chunk][out channel][8].  One thread issues the
// 25 * (channels / 16) tcgen05.mma instructions (kind::f16, BF16 x BF16 ->
// FP32 in tensor memory), commits them to an mbarrier, and the four warps
// read the 128 x N accumulator back with tcgen05.ld (warp w owns lanes
// 32w..32w+31, i.e. pixels 32w..32w+31) for the epilogue: bias + ReLU ->
// BF16 activations, bias -> FP32 outputs, or (input-gradient pass) the ReLU
// mask of the forward activation.
//
// Every wait is bounded: an mbarrier that does not complete within ~2 s of
// polling sets the network's error flag; the CTA then waits once more (also
// bounded) and releases its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "../../include/ouc.h"
#include "../../include/ouc_corrector.h"

namespace ouc {
namespace cnn {

using bf16 = __nv_bfloat16;

constexpr int kTile = 128;            // GEMM M: pixels per tile
constexpr int kPC = kTile + 4;        // patch columns (2 + 2 halo)
constexpr int kTaps = 25;
constexpr int kMaxPairs = 32 * 32;     // (cin, cout) pairs of the widest layer
constexpr int kMaxRowBlocks = 64;      // CTAs (partial-sum slots) of k_wgrad_tc
constexpr int kBgradBlocks = 256;      // blocks of k_bgrad (8 warps each)
constexpr int kThreadsConv = 128;

struct LayerDims {
    int cin, cout, cin_pad, cout_pad;
};
constexpr LayerDims kL[4] = {{OUC_CNN_IN, OUC_CNN_WIDTH, 16, 32},
                             {OUC_CNN_WIDTH, OUC_CNN_WIDTH, 32, 32},
                             {OUC_CNN_WIDTH, OUC_CNN_WIDTH, 32, 32},
                             {OUC_CNN_WIDTH, OUC_CNN_OUT, 32, 16}};

constexpr int w_count(int l) { return kL[l].cout * kL[l].cin * kTaps; }
constexpr int p_offset(int l) { return l == 0 ? 0 : p_offset(l - 1) + w_count(l - 1) + kL[l - 1].cout; }
constexpr int kNParams = p_offset(3) + w_count(3) + kL[3].cout;

// ---- PTX helpers (tcgen05, mbarrier) ---------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle, K-major canonical layout:
// start address, leading-dimension byte offset (between the two 8-element K
// chunks), stride byte offset (between 8-row groups), all >> 4; version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Poll with back-off; false after ~2^24 polls (well over a second).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < (1 << 24); ++i) {
        if (mbar_test(bar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// The wait takes the loaded registers as operands, so that no use of them can
// be scheduled before it.
#define OUC_R16(r, o)                                                                                               \
    "+r"(r[o + 0]), "+r"(r[o + 1]), "+r"(r[o + 2]), "+r"(r[o + 3]), "+r"(r[o + 4]), "+r"(r[o + 5]), "+r"(r[o + 6]), \
        "+r"(r[o + 7]), "+r"(r[o + 8]), "+r"(r[o + 9]), "+r"(r[o + 10]), "+r"(r[o + 11]), "+r"(r[o + 12]),          \
        "+r"(r[o + 13]), "+r"(r[o + 14]), "+r"(r[o + 15])

template <int NC>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[NC]) {
    static_assert(NC == 16 || NC == 32, "16 or 32 columns");
    uint32_t q0[16], q1[16];
    tmem_ld16(taddr, q0);
    if (NC == 32) tmem_ld16(taddr + 16, q1);
    asm volatile("tcgen05.wait::ld.sync.aligned;" : OUC_R16(q0, 0)::"memory");
    if (NC == 32) asm volatile("" : OUC_R16(q1, 0));
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        r[k] = q0[k];
        if (NC == 32) r[16 + k] = q1[k];
    }
}

// ---- convolution kernel ----------------------------------------------------

enum Epi : int { kHidden = 0, kOut = 1, kDgrad = 2 };

struct ConvArgs {
    int n, H, W;
    const bf16* x;        // [n][H][W][CIN]
    const bf16* w;        // packed [tap][CIN / 8][COUT][8]
    const float* bias;    // [COUT] or null
    const bf16* mask;     // kDgrad: forward activation [n][H][W][COUT]
    void* y;              // bf16 [n][H][W][COUT] (kHidden, kDgrad) or float [n][H][W][cout_real] (kOut)
    int cout_real;
    int* err;
};

template <int CIN, int COUT>
struct ConvGeo {
    static constexpr int NQ = CIN / 8;
    static constexpr int w_bytes = kTaps * CIN * COUT * 2;
    static constexpr int p_bytes = 5 * NQ * kPC * 16;
    static constexpr int bytes = w_bytes + p_bytes;
};

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kThreadsConv) k_conv5(const ConvArgs a) {
    using G = ConvGeo<CIN, COUT>;
    constexpr int NQ = G::NQ;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* s_w = smem;
    uint8_t* s_p = smem + G::w_bytes;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < G::w_bytes / 16; i += kThreadsConv)
        reinterpret_cast<uint4*>(s_w)[i] = reinterpret_cast<const uint4*>(a.w)[i];
    if (tid == 0) mbar_init(&bar, 1);
    __syncwarp();   // .sync.aligned tcgen05 instructions need a converged warp
    if (warp == 0) tmem_alloc(&tmem_base, 32);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const int tiles_w = (a.W + kTile - 1) / kTile;
    const int ntiles = a.n * a.H * tiles_w;
    uint32_t phase = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int tw = tile % tiles_w, row = tile / tiles_w;
        const int img = row / a.H, h = row - img * a.H;
        const int z0 = tw * kTile;
        // input patch: rows h-2..h+2, columns z0-2..z0+129, zero outside the image
        for (int i = tid; i < 5 * kPC * NQ; i += kThreadsConv) {
            const int q = i % NQ, rest = i / NQ, c = rest % kPC, r = rest / kPC;
            const int gh = h + r - 2, gz = z0 + c - 2;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gh >= 0 && gh < a.H && gz >= 0 && gz < a.W)
                v = *reinterpret_cast<const uint4*>(a.x + (((size_t)img * a.H + gh) * a.W + gz) * CIN + q * 8);
            *reinterpret_cast<uint4*>(s_p + ((size_t)(r * NQ + q) * kPC + c) * 16) = v;
        }
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t pb = smem_u32(s_p), wb = smem_u32(s_w);
            constexpr uint32_t idesc = idesc_bf16(kTile, COUT);
            uint32_t acc = 0;
#pragma unroll 1
            for (int dx = 0; dx < 5; ++dx) {
#pragma unroll 1
                for (int dz = 0; dz < 5; ++dz) {
#pragma unroll
                    for (int ks = 0; ks < NQ / 2; ++ks) {
                        const uint32_t tap = dx * 5 + dz;
                        const uint64_t ad = umma_desc(pb + ((dx * NQ + 2 * ks) * kPC + dz) * 16, kPC * 16, 128);
                        const uint64_t bd = umma_desc(wb + ((tap * NQ + 2 * ks) * COUT) * 16, COUT * 16, 128);
                        umma_bf16(tmem, ad, bd, idesc, acc);
                        acc = 1;
                    }
                }
            }
            umma_commit(&bar);
        }
        const bool done = mbar_wait(&bar, phase);
        phase ^= 1u;
        if (!__syncthreads_and(done)) {
            if (tid == 0) atomicExch(a.err, 1);
            mbar_wait(&bar, phase ^ 1u);   // one more bounded wait for the MMAs in flight
            break;
        }
        tc_fence_after();
        uint32_t r[COUT];
        __syncwarp();
        tmem_ld<COUT>(tmem + ((uint32_t)(warp * 32) << 16), r);
        const int gz = z0 + warp * 32 + lane;
        if (gz < a.W) {
            const size_t p = ((size_t)img * a.H + h) * a.W + gz;
            if (EPI == kOut) {
                float* y = static_cast<float*>(a.y) + p * a.cout_real;
#pragma unroll
                for (int c = 0; c < COUT; ++c)
                    if (c < a.cout_real) y[c] = __uint_as_float(r[c]) + a.bias[c];
            } else {
                uint4* y = reinterpret_cast<uint4*>(static_cast<bf16*>(a.y) + p * COUT);
                const uint4* mk = EPI == kDgrad ? reinterpret_cast<const uint4*>(a.mask + p * COUT) : nullptr;
#pragma unroll
                for (int c8 = 0; c8 < COUT / 8; ++c8) {
                    __align__(16) bf16 o[8];
                    __align__(16) bf16 mv[8];
                    if (EPI == kDgrad) *reinterpret_cast<uint4*>(mv) = mk[c8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const int c = 8 * c8 + k;
                        float v = __uint_as_float(r[c]);
                        if (EPI == kHidden) v = fmaxf(v + a.bias[c], 0.f);
                        else v = __bfloat162float(mv[k]) > 0.f ? v : 0.f;
                        o[k] = __float2bfloat16_rn(v);
                    }
                    y[c8] = *reinterpret_cast<const uint4*>(o);
                }
            }
        }
        tc_fence_before();
        __syncthreads();   // accumulator read and patch consumed before the next tile
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    __syncwarp();
    if (warp == 0) tmem_dealloc(tmem, 32);
}

template <int CIN, int COUT, int EPI>
cudaError_t launch_conv(const ConvArgs& a, int sms, cudaStream_t s) {
    constexpr int bytes = ConvGeo<CIN, COUT>::bytes;
    // the shared-memory opt-in is a per-device setting: set on the current
    // device at every launch (a host-side call; a few launches per step);
    // if it is refused nothing is launched and the caller reports it
    const cudaError_t e = cudaFuncSetAttribute(k_conv5<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               bytes);
    if (e != cudaSuccess) return e;
    const int tiles = a.n * a.H * ((a.W + kTile - 1) / kTile);
    const int grid = tiles < 2 * sms ? tiles : 2 * sms;
    k_conv5<CIN, COUT, EPI><<<grid, kThreadsConv, bytes, s>>>(a);
    return cudaSuccess;
}

// ---- weight gradients on the tensor cores ------------------------------------
//
// dW[tap][co][ci] = sum_p X[p + s(tap)][ci] G[p][co] over all pixels p, with
// s(dx, dz) = (dx - 2, dz - 2).  The pixels are the GEMM's K dimension, so
// the operand that carries the tap shift must move along K by whole 16-byte
// rows: both operands use the no-swizzle MN-major layout, in which K
// advances 16 bytes per pixel.  Per 128-pixel tile (one image row, as in
// k_conv5) the CTA stages
//   * the input patch, rows h-2..h+2 (plus zero rows up to 8) and columns
//     z0-2..z0+129, as [row][channel chunk of 8][column][8 channels] -- the
//     layout of k_conv5 -- so that M = 128 consecutive 8-channel groups are
//     (row, chunk) pairs at one uniform stride: 4 rows x 32 channels (or 8 x
//     16), and the tap shift dz is a start offset of 16 dz bytes;
//   * the output gradient of the tile, [chunk of 8 output channels][pixel]
//     [8 channels], the N operand;
// and one thread issues, for each dz and row group, 8 MMAs of K = 16
// (kind::f16, BF16 inputs, FP32 accumulation in tensor memory): D[(dx, ci)]
// [co] for the tile's pixels, accumulated over all of the CTA's tiles.  At
// the end each warp reads its 32 accumulator lanes (rows (dx, ci)) and
// writes the CTA's partial sums, which k_wgrad_sum adds in CTA order: the
// result does not depend on scheduling, so training repeats bit for bit.
template <int CIN, int COUT>
struct WgradGeo {
    static constexpr int NQ = CIN / 8;                  // input-channel chunks
    static constexpr int RPG = 128 / CIN;               // patch rows per M = 128 row group
    static constexpr int NRG = (5 + RPG - 1) / RPG;     // row groups covering dx = 0..4
    static constexpr int PR = NRG * RPG;                // patch rows held (rows >= 5 stay zero)
    static constexpr int p_bytes = PR * NQ * kPC * 16;
    static constexpr int g_bytes = (COUT / 8) * kTile * 16;
    static constexpr int bytes = p_bytes + g_bytes;
    static constexpr int ncols = 5 * NRG * COUT;        // accumulator columns
    static constexpr int tmem_cols = ncols <= 32 ? 32 : ncols <= 64 ? 64 : ncols <= 128 ? 128 : ncols <= 256 ? 256 : 512;
    static_assert(ncols <= 512, "accumulators fit tensor memory");
};

// Instruction descriptor as idesc_bf16 with both operands MN-major
// (bit 15: A, bit 16: B).
__host__ __device__ constexpr uint32_t idesc_bf16_mn(int M, int N) { return idesc_bf16(M, N) | (1u << 15) | (1u << 16); }

// No-swizzle MN-major descriptor: 8 K rows of 16 bytes per core matrix, K
// groups of 8 rows at `kgroup` bytes, M/N groups of 8 elements at `mgroup`
// bytes (leading-dimension offset = K-group stride, stride offset = M/N
// group stride for this layout).
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr, uint32_t kgroup, uint32_t mgroup) {
    return umma_desc(saddr, kgroup, mgroup);
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreadsConv) k_wgrad_tc(int n, int H, int W, const bf16* x, const bf16* g,
                                                        int cin_real, int cout_real, float* part, int* err) {
    using G = WgradGeo<CIN, COUT>;
    constexpr int NQ = G::NQ, NRG = G::NRG, PR = G::PR, QO = COUT / 8;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* s_p = smem;
    uint8_t* s_g = smem + G::p_bytes;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // patch rows 5 .. PR-1 are read by the last row group's MMAs and stay zero
    for (int i = tid; i < (PR - 5) * NQ * kPC; i += kThreadsConv)
        reinterpret_cast<uint4*>(s_p + 5 * NQ * kPC * 16)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) mbar_init(&bar, 1);
    __syncwarp();
    if (warp == 0) tmem_alloc(&tmem_base, G::tmem_cols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const int tiles_w = (W + kTile - 1) / kTile;
    const int ntiles = n * H * tiles_w;
    uint32_t phase = 0, acc = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int tw = tile % tiles_w, row = tile / tiles_w;
        const int img = row / H, h = row - img * H;
        const int z0 = tw * kTile;
        for (int i = tid; i < 5 * kPC * NQ; i += kThreadsConv) {
            const int q = i % NQ, rest = i / NQ, c = rest % kPC, r = rest / kPC;
            const int gh = h + r - 2, gz = z0 + c - 2;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gh >= 0 && gh < H && gz >= 0 && gz < W)
                v = *reinterpret_cast<const uint4*>(x + (((size_t)img * H + gh) * W + gz) * CIN + q * 8);
            *reinterpret_cast<uint4*>(s_p + ((size_t)(r * NQ + q) * kPC + c) * 16) = v;
        }
        for (int i = tid; i < kTile * QO; i += kThreadsConv) {
            const int q = i % QO, c = i / QO, gz = z0 + c;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);   // pixels beyond the row add nothing
            if (gz < W) v = *reinterpret_cast<const uint4*>(g + (((size_t)img * H + h) * W + gz) * COUT + q * 8);
            *reinterpret_cast<uint4*>(s_g + ((size_t)q * kTile + c) * 16) = v;
        }
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t pb = smem_u32(s_p), gb = smem_u32(s_g);
            constexpr uint32_t idesc = idesc_bf16_mn(128, COUT);
#pragma unroll 1
            for (int dz = 0; dz < 5; ++dz) {
#pragma unroll 1
                for (int rg = 0; rg < NRG; ++rg) {
                    const uint32_t d = tmem + (uint32_t)((dz * NRG + rg) * COUT);
#pragma unroll
                    for (int ks = 0; ks < kTile / 16; ++ks) {
                        const uint64_t ad = umma_desc_mn(pb + ((rg * G::RPG * NQ) * kPC + dz + 16 * ks) * 16, 128,
                                                         kPC * 16);
                        const uint64_t bd = umma_desc_mn(gb + (16 * ks) * 16, 128, kTile * 16);
                        umma_bf16(d, ad, bd, idesc, (acc | (uint32_t)ks) ? 1u : 0u);
                    }
                }
            }
            umma_commit(&bar);
        }
        acc = 1;
        const bool done = mbar_wait(&bar, phase);
        phase ^= 1u;
        if (!__syncthreads_and(done)) {
            if (tid == 0) atomicExch(err, 1);
            mbar_wait(&bar, phase ^ 1u);   // one more bounded wait for the MMAs in flight
            ok = false;
            break;
        }
    }
    tc_fence_after();
    // accumulator row m = 32 warp + lane: 8-channel group j = m / 8 = (row in
    // group, chunk), channel e = m % 8; column (dz, rg) * COUT + co
    if (ok) {
        const int m = warp * 32 + lane, j = m >> 3, e = m & 7;
        const int ci = (j % NQ) * 8 + e;
#pragma unroll 1
        for (int dz = 0; dz < 5; ++dz) {
#pragma unroll 1
            for (int rg = 0; rg < NRG; ++rg) {
                uint32_t r[COUT];
                __syncwarp();
                tmem_ld<COUT>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((dz * NRG + rg) * COUT), r);
                const int dx = rg * G::RPG + j / NQ;
                if (dx < 5 && ci < cin_real) {
                    const int tap = dx * 5 + dz;
                    float* out = part + ((size_t)blockIdx.x * kTaps + tap) * kMaxPairs;
#pragma unroll
                    for (int co = 0; co < COUT; ++co)
                        if (co < cout_real) out[co * cin_real + ci] = __uint_as_float(r[co]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    __syncwarp();
    if (warp == 0) tmem_dealloc(tmem, G::tmem_cols);
}

template <int CIN, int COUT>
cudaError_t launch_wgrad(int n, int H, int W, const bf16* x, const bf16* g, int cin_real, int cout_real, float* part,
                         int* err, int* nblocks, cudaStream_t s) {
    constexpr int bytes = WgradGeo<CIN, COUT>::bytes;
    const cudaError_t e = cudaFuncSetAttribute(k_wgrad_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    const int tiles = n * H * ((W + kTile - 1) / kTile);
    // a fixed grid (at most kMaxRowBlocks partial-sum slots), independent of the device
    const int grid = tiles < kMaxRowBlocks ? tiles : kMaxRowBlocks;
    k_wgrad_tc<CIN, COUT><<<grid, kThreadsConv, bytes, s>>>(n, H, W, x, g, cin_real, cout_real, part, err);
    *nblocks = grid;
    return cudaSuccess;
}

// ---- gradient sums, bias gradients, packing, Adam ---------------------------

// dw[co][ci][tap] += sum over the CTAs' partial sums, in CTA order.
__global__ void k_wgrad_sum(int nblocks, int cin_real, int cout_real, const float* part, float* dw) {
    const int npairs = cin_real * cout_real;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < kTaps * npairs; i += blockDim.x * gridDim.x) {
        const int tap = i / npairs, pr = i - tap * npairs;
        float s = 0.f;
        for (int b = 0; b < nblocks; ++b) s += part[((size_t)b * kTaps + tap) * kMaxPairs + pr];
        const int ci = pr % cin_real, co = pr / cin_real;
        dw[((size_t)co * cin_real + ci) * kTaps + tap] += s;
    }
}

template <int COUT>
__global__ void k_bgrad(size_t npix, const bf16* g, int cout_real, float* part) {
    float acc[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) acc[c] = 0.f;
    for (size_t p = threadIdx.x + (size_t)blockIdx.x * blockDim.x; p < npix; p += (size_t)blockDim.x * gridDim.x)
#pragma unroll
        for (int c = 0; c < COUT; ++c) acc[c] += __bfloat162float(g[p * COUT + c]);
    const int wid = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    for (int c = 0; c < cout_real; ++c) {
        float v = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) part[(size_t)wid * 32 + c] = v;   // one slot per warp and channel
    }
}

// db[c] += sum over the warps' partial sums, in warp order.
__global__ void k_bgrad_sum(int nwarps, int cout_real, const float* part, float* db) {
    const int c = threadIdx.x;
    if (c >= cout_real) return;
    float s = 0.f;
    for (int w = 0; w < nwarps; ++w) s += part[(size_t)w * 32 + c];
    db[c] += s;
}

// float [P][creal] -> bf16 [P][cpad], zero-padded channels
__global__ void k_to_bf16(size_t npix, int creal, int cpad, const float* in, bf16* out) {
    for (size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x; i < npix * cpad; i += (size_t)blockDim.x * gridDim.x) {
        const size_t p = i / cpad;
        const int c = (int)(i % cpad);
        out[i] = __float2bfloat16_rn(c < creal ? in[p * creal + c] : 0.f);
    }
}

// Pack W[cout][cin][5][5] (FP32) into the B-operand layout [tap][cin_pad/8][cout_pad][8]
// (forward), or, transposed and flipped, into the input-gradient weights
// W'[tap'][cout_pad/8][cin_pad][8] with W'[ci][co][tap'] = W[co][ci][24 - tap'].
__global__ void k_pack(const float* w, int cin, int cout, int cin_pad, int cout_pad, bool dgrad, bf16* out) {
    const int kin = dgrad ? cout_pad : cin_pad, kout = dgrad ? cin_pad : cout_pad;
    const int total = kTaps * kin * kout;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < total; i += blockDim.x * gridDim.x) {
        const int e = i % 8, rest = i / 8, o = rest % kout, rest2 = rest / kout, q = rest2 % (kin / 8),
                  tap = rest2 / (kin / 8);
        const int k = q * 8 + e;   // input channel of this (possibly transposed) convolution
        float v = 0.f;
        if (!dgrad) {
            if (k < cin && o < cout) v = w[((size_t)o * cin + k) * kTaps + tap];
        } else {
            if (k < cout && o < cin) v = w[((size_t)k * cin + o) * kTaps + (kTaps - 1 - tap)];
        }
        out[i] = __float2bfloat16_rn(v);
    }
}

__global__ void k_adam(int n, float* p, const float* g, float* m, float* v, float lr_t, float b1, float b2, float eps) {
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < n; i += blockDim.x * gridDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr_t * mi / (sqrtf(vi) + eps);
    }
}

// Masked mean squared error of n images [n][H][W][8] against targets:
// g = 2 (y - t) / count on the rectangle [i0, i1) x [j0, j1) of every image
// and 0 elsewhere; loss += sum (y - t)^2 / count.
__global__ void k_mse(int n, int H, int W, int i0, int i1, int j0, int j1, float inv_count, const float* y,
                      const float* t, float* g, double* loss) {
    double acc = 0.0;
    const size_t P = (size_t)n * H * W;
    for (size_t p = threadIdx.x + (size_t)blockIdx.x * blockDim.x; p < P; p += (size_t)blockDim.x * gridDim.x) {
        const int j = (int)(p % W), i = (int)((p / W) % H);
        const bool in = i >= i0 && i < i1 && j >= j0 && j < j1;
#pragma unroll
        for (int c = 0; c < OUC_CNN_OUT; ++c) {
            const float d = in ? y[p * OUC_CNN_OUT + c] - t[p * OUC_CNN_OUT + c] : 0.f;
            g[p * OUC_CNN_OUT + c] = 2.f * d * inv_count;
            acc += (double)d * d;
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc * inv_count);
}

}  // namespace cnn
}  // namespace ouc

using namespace ouc::cnn;

struct ouc_cnn {
    int device = 0;
    int sms = 148;
    float* params = nullptr;     // FP32 master [kNParams]
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    long long adam_t = 0;
    bf16* wf[4] = {};            // packed forward weights
    bf16* wd[4] = {};            // packed input-gradient weights (layers 1..3)
    int* err = nullptr;
    float* part = nullptr;       // gradient partial sums, reduced in a fixed order (kMaxRowBlocks x 25 x kMaxPairs)
    // activations of the last forward
    int n = 0, H = 0, W = 0;
    size_t cap = 0;              // pixels the buffers hold
    bf16* x0 = nullptr;          // [P][16]
    bf16* y[3] = {};             // [P][32]
    bf16* g16 = nullptr;         // [P][16]  output-layer gradient
    bf16* g[2] = {};             // [P][32]
};

namespace {

int repack(ouc_cnn* net, cudaStream_t s) {
    for (int l = 0; l < 4; ++l) {
        const LayerDims d = kL[l];
        const float* w = net->params + p_offset(l);
        k_pack<<<64, 256, 0, s>>>(w, d.cin, d.cout, d.cin_pad, d.cout_pad, false, net->wf[l]);
        if (l > 0) k_pack<<<64, 256, 0, s>>>(w, d.cin, d.cout, d.cin_pad, d.cout_pad, true, net->wd[l]);
    }
    return cudaGetLastError() == cudaSuccess ? OUC_OK : OUC_ECUDA;
}

int ensure_acts(ouc_cnn* net, size_t P) {
    if (P <= net->cap) return OUC_OK;
    cudaFree(net->x0); cudaFree(net->g16);
    for (auto& p : net->y) cudaFree(p);
    for (auto& p : net->g) cudaFree(p);
    net->cap = 0;
    bool ok = cudaMalloc(&net->x0, P * 16 * 2) == cudaSuccess && cudaMalloc(&net->g16, P * 16 * 2) == cudaSuccess;
    for (auto& p : net->y) ok = ok && cudaMalloc(&p, P * 32 * 2) == cudaSuccess;
    for (auto& p : net->g) ok = ok && cudaMalloc(&p, P * 32 * 2) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return OUC_ENOMEM;
    }
    net->cap = P;
    return OUC_OK;
}

}  // namespace

extern "C" {

int ouc_cnn_nparams(void) { return kNParams; }

int ouc_cnn_create(int device, ouc_cnn** out) {
    if (!out) return OUC_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return OUC_ENODEV;
    }
    cudaDeviceProp prop;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess ||
        prop.major != 10)
        return OUC_ENODEV;
    ouc_cnn* net = new (std::nothrow) ouc_cnn();
    if (!net) return OUC_ENOMEM;
    net->device = device;
    net->sms = prop.multiProcessorCount;
    const size_t pb = (size_t)kNParams * 4;
    bool ok = cudaMalloc(&net->params, pb) == cudaSuccess && cudaMalloc(&net->grads, pb) == cudaSuccess &&
              cudaMalloc(&net->adam_m, pb) == cudaSuccess && cudaMalloc(&net->adam_v, pb) == cudaSuccess &&
              cudaMalloc(&net->err, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&net->part, (size_t)kMaxRowBlocks * kTaps * kMaxPairs * sizeof(float)) == cudaSuccess;
    for (int l = 0; l < 4 && ok; ++l) {
        ok = cudaMalloc(&net->wf[l], (size_t)kTaps * kL[l].cin_pad * kL[l].cout_pad * 2) == cudaSuccess;
        if (ok && l > 0) ok = cudaMalloc(&net->wd[l], (size_t)kTaps * kL[l].cin_pad * kL[l].cout_pad * 2) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        ouc_cnn_destroy(net);
        return OUC_ENOMEM;
    }
    cudaMemset(net->params, 0, pb);
    cudaMemset(net->grads, 0, pb);
    cudaMemset(net->adam_m, 0, pb);
    cudaMemset(net->adam_v, 0, pb);
    cudaMemset(net->err, 0, sizeof(int));
    if (repack(net, nullptr) || cudaDeviceSynchronize() != cudaSuccess) {
        ouc_cnn_destroy(net);
        return OUC_ECUDA;
    }
    *out = net;
    return OUC_OK;
}

int ouc_cnn_destroy(ouc_cnn* net) {
    if (!net) return OUC_OK;
    cudaSetDevice(net->device);
    cudaDeviceSynchronize();
    cudaFree(net->params); cudaFree(net->grads); cudaFree(net->adam_m); cudaFree(net->adam_v); cudaFree(net->err); cudaFree(net->part);
    for (auto* p : net->wf) cudaFree(p);
    for (auto* p : net->wd) cudaFree(p);
    cudaFree(net->x0); cudaFree(net->g16);
    for (auto* p : net->y) cudaFree(p);
    for (auto* p : net->g) cudaFree(p);
    delete net;
    return OUC_OK;
}

int ouc_cnn_set_params(ouc_cnn* net, const float* params) {
    if (!net || !params) return OUC_EINVAL;
    cudaSetDevice(net->device);
    if (cudaMemcpy(net->params, params, (size_t)kNParams * 4, cudaMemcpyHostToDevice) != cudaSuccess) return OUC_ECUDA;
    if (repack(net, nullptr)) return OUC_ECUDA;
    return cudaDeviceSynchronize() == cudaSuccess ? OUC_OK : OUC_ECUDA;
}

int ouc_cnn_get_params(const ouc_cnn* net, float* params) {
    if (!net || !params) return OUC_EINVAL;
    cudaSetDevice(net->device);
    return cudaMemcpy(params, net->params, (size_t)kNParams * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? OUC_OK
                                                                                                      : OUC_ECUDA;
}

int ouc_cnn_forward_dev(ouc_cnn* net, int n, int H, int W, const float* d_in, float* d_out, void* stream) {
    if (!net || !d_in || !d_out || n < 1 || H < 1 || W < 1) return OUC_EINVAL;
    cudaSetDevice(net->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t P = (size_t)n * H * W;
    if (ensure_acts(net, P)) return OUC_ENOMEM;
    net->n = n; net->H = H; net->W = W;
    k_to_bf16<<<1024, 256, 0, s>>>(P, OUC_CNN_IN, 16, d_in, net->x0);
    ConvArgs a{};
    a.n = n; a.H = H; a.W = W; a.err = net->err;
    a.x = net->x0; a.w = net->wf[0]; a.bias = net->params + p_offset(0) + w_count(0); a.y = net->y[0];
    if (launch_conv<16, 32, kHidden>(a, net->sms, s) != cudaSuccess) return OUC_ECUDA;
    for (int l = 1; l < 3; ++l) {
        a.x = net->y[l - 1]; a.w = net->wf[l]; a.bias = net->params + p_offset(l) + w_count(l); a.y = net->y[l];
        if (launch_conv<32, 32, kHidden>(a, net->sms, s) != cudaSuccess) return OUC_ECUDA;
    }
    a.x = net->y[2]; a.w = net->wf[3]; a.bias = net->params + p_offset(3) + w_count(3); a.y = d_out;
    a.cout_real = OUC_CNN_OUT;
    if (launch_conv<32, 16, kOut>(a, net->sms, s) != cudaSuccess) return OUC_ECUDA;
    return cudaGetLastError() == cudaSuccess ? OUC_OK : OUC_ECUDA;
}

int ouc_cnn_backward_dev(ouc_cnn* net, const float* d_gout, void* stream) {
    if (!net || !d_gout) return OUC_EINVAL;
    if (net->n == 0) return OUC_ESTATE;
    cudaSetDevice(net->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int n = net->n, H = net->H, W = net->W;
    const size_t P = (size_t)n * H * W;
    int nb = 0;   // CTAs of the weight-gradient launch: partial-sum slots to add
    k_to_bf16<<<1024, 256, 0, s>>>(P, OUC_CNN_OUT, 16, d_gout, net->g16);
    // layer 4: weights and bias, then the gradient into layer 3's output
    float* gp = net->grads;
    if (launch_wgrad<32, 16>(n, H, W, net->y[2], net->g16, kL[3].cin, kL[3].cout, net->part, net->err, &nb, s) !=
        cudaSuccess)
        return OUC_ECUDA;
    k_wgrad_sum<<<64, 256, 0, s>>>(nb, kL[3].cin, kL[3].cout, net->part, gp + p_offset(3));
    k_bgrad<16><<<kBgradBlocks, 256, 0, s>>>(P, net->g16, kL[3].cout, net->part);
    k_bgrad_sum<<<1, 32, 0, s>>>(kBgradBlocks * 8, kL[3].cout, net->part, gp + p_offset(3) + w_count(3));
    ConvArgs a{};
    a.n = n; a.H = H; a.W = W; a.err = net->err;
    a.x = net->g16; a.w = net->wd[3]; a.mask = net->y[2]; a.y = net->g[0];
    if (launch_conv<16, 32, kDgrad>(a, net->sms, s) != cudaSuccess) return OUC_ECUDA;
    // layers 3 and 2
    for (int l = 2; l >= 1; --l) {
        const bf16* gl = net->g[(2 - l) & 1];
        if (launch_wgrad<32, 32>(n, H, W, net->y[l - 1], gl, kL[l].cin, kL[l].cout, net->part, net->err, &nb, s) !=
            cudaSuccess)
            return OUC_ECUDA;
        k_wgrad_sum<<<64, 256, 0, s>>>(nb, kL[l].cin, kL[l].cout, net->part, gp + p_offset(l));
        k_bgrad<32><<<kBgradBlocks, 256, 0, s>>>(P, gl, kL[l].cout, net->part);
        k_bgrad_sum<<<1, 32, 0, s>>>(kBgradBlocks * 8, kL[l].cout, net->part, gp + p_offset(l) + w_count(l));
        a.x = gl; a.w = net->wd[l]; a.mask = net->y[l - 1]; a.y = net->g[(3 - l) & 1];
        if (launch_conv<32, 32, kDgrad>(a, net->sms, s) != cudaSuccess) return OUC_ECUDA;
    }
    // layer 1
    const bf16* g1 = net->g[0];
    if (launch_wgrad<16, 32>(n, H, W, net->x0, g1, kL[0].cin, kL[0].cout, net->part, net->err, &nb, s) != cudaSuccess)
        return OUC_ECUDA;
    k_wgrad_sum<<<64, 256, 0, s>>>(nb, kL[0].cin, kL[0].cout, net->part, gp + p_offset(0));
    k_bgrad<32><<<kBgradBlocks, 256, 0, s>>>(P, g1, kL[0].cout, net->part);
    k_bgrad_sum<<<1, 32, 0, s>>>(kBgradBlocks * 8, kL[0].cout, net->part, gp + p_offset(0) + w_count(0));
    return cudaGetLastError() == cudaSuccess ? OUC_OK : OUC_ECUDA;
}

int ouc_cnn_zero_grad(ouc_cnn* net, void* stream) {
    if (!net) return OUC_EINVAL;
    cudaSetDevice(net->device);
    return cudaMemsetAsync(net->grads, 0, (size_t)kNParams * 4, (cudaStream_t)stream) == cudaSuccess ? OUC_OK
                                                                                                      : OUC_ECUDA;
}

int ouc_cnn_get_grads(const ouc_cnn* net, float* grads) {
    if (!net || !grads) return OUC_EINVAL;
    cudaSetDevice(net->device);
    return cudaMemcpy(grads, net->grads, (size_t)kNParams * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? OUC_OK
                                                                                                    : OUC_ECUDA;
}

int ouc_cnn_adam_step(ouc_cnn* net, float lr, float beta1, float beta2, float eps, void* stream) {
    if (!net || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0)) return OUC_EINVAL;
    cudaSetDevice(net->device);
    cudaStream_t s = (cudaStream_t)stream;
    ++net->adam_t;
    const double c1 = 1.0 - std::pow((double)beta1, (double)net->adam_t);
    const double c2 = 1.0 - std::pow((double)beta2, (double)net->adam_t);
    const float lr_t = (float)(lr * std::sqrt(c2) / c1);
    k_adam<<<64, 256, 0, s>>>(kNParams, net->params, net->grads, net->adam_m, net->adam_v, lr_t, beta1, beta2, eps);
    return repack(net, s);
}

int ouc_cnn_train(ouc_cnn* net, const float* d_in, const float* d_tgt, int npairs, int H, int W, int i0, int i1, int j0,
                  int j1, int batch, int epochs, float lr, unsigned seed, float* epoch_loss, void* stream) {
    if (!net || !d_in || !d_tgt || npairs < 1 || H < 1 || W < 1 || batch < 1 || epochs < 1 || !(lr > 0)) return OUC_EINVAL;
    if (!(0 <= i0 && i0 < i1 && i1 <= H && 0 <= j0 && j0 < j1 && j1 <= W)) return OUC_EINVAL;
    cudaSetDevice(net->device);
    cudaStream_t s = (cudaStream_t)stream;
    batch = std::min(batch, npairs);
    const size_t img = (size_t)H * W;
    float *bin = nullptr, *btg = nullptr, *by = nullptr, *bg = nullptr;
    double* dloss = nullptr;
    bool ok = cudaMalloc(&bin, batch * img * OUC_CNN_IN * 4) == cudaSuccess &&
              cudaMalloc(&btg, batch * img * OUC_CNN_OUT * 4) == cudaSuccess &&
              cudaMalloc(&by, batch * img * OUC_CNN_OUT * 4) == cudaSuccess &&
              cudaMalloc(&bg, batch * img * OUC_CNN_OUT * 4) == cudaSuccess &&
              cudaMalloc(&dloss, sizeof(double)) == cudaSuccess;
    int rc = ok ? OUC_OK : OUC_ENOMEM;
    std::vector<int> order(npairs);
    for (int k = 0; k < npairs; ++k) order[k] = k;
    std::mt19937 rng(seed);
    const int nb = (npairs + batch - 1) / batch;
    for (int e = 0; e < epochs && rc == OUC_OK; ++e) {
        std::shuffle(order.begin(), order.end(), rng);
        cudaMemsetAsync(dloss, 0, sizeof(double), s);
        for (int b = 0; b < nb && rc == OUC_OK; ++b) {
            const int n = std::min(batch, npairs - b * batch);
            for (int k = 0; k < n; ++k) {
                const size_t q = order[b * batch + k];
                cudaMemcpyAsync(bin + k * img * OUC_CNN_IN, d_in + q * img * OUC_CNN_IN, img * OUC_CNN_IN * 4,
                                cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(btg + k * img * OUC_CNN_OUT, d_tgt + q * img * OUC_CNN_OUT, img * OUC_CNN_OUT * 4,
                                cudaMemcpyDeviceToDevice, s);
            }
            if ((rc = ouc_cnn_forward_dev(net, n, H, W, bin, by, s))) break;
            const float inv = 1.f / ((float)n * (i1 - i0) * (j1 - j0) * OUC_CNN_OUT);
            k_mse<<<592, 256, 0, s>>>(n, H, W, i0, i1, j0, j1, inv, by, btg, bg, dloss);
            if ((rc = ouc_cnn_zero_grad(net, s)) || (rc = ouc_cnn_backward_dev(net, bg, s))) break;
            // bias-free network: a zero input gives a zero output
            for (int l = 0; l < 4; ++l)
                cudaMemsetAsync(net->grads + p_offset(l) + w_count(l), 0, kL[l].cout * sizeof(float), s);
            if ((rc = ouc_cnn_adam_step(net, lr, 0.9f, 0.999f, 1e-8f, s))) break;
        }
        double l = 0;
        if (rc == OUC_OK && cudaMemcpyAsync(&l, dloss, sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
            cudaStreamSynchronize(s) == cudaSuccess) {
            if (epoch_loss) epoch_loss[e] = (float)(l / nb);
        } else if (rc == OUC_OK) {
            rc = OUC_ECUDA;
        }
    }
    cudaStreamSynchronize(s);
    cudaFree(bin); cudaFree(btg); cudaFree(by); cudaFree(bg); cudaFree(dloss);
    if (rc == OUC_OK && cudaGetLastError() != cudaSuccess) rc = OUC_ECUDA;
    return rc;
}

int ouc_cnn_error(ouc_cnn* net) {
    if (!net) return OUC_EINVAL;
    cudaSetDevice(net->device);
    int e = 0;
    cudaMemcpy(&e, net->err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemset(net->err, 0, sizeof(int));
    return e;
}

}  // extern "C"
