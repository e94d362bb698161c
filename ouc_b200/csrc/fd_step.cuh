// Fused time-step kernel of the elastic P/S-decoupled staggered-grid
// scheme (sm_100a).
//
// One launch advances one wavefield per shot of a batch by one time step.
// The reference does it in two launches that talk through six full-grid
// HBM arrays (forward_s then forward_u, PS:2261-2264; rt_s_res/rt_u_res;
// reshot_u/reshot_s).  Here each CTA owns a TX x TZ tile of one shot
// (blockIdx.y = shot) and, in three phases separated by __syncthreads():
//   1. brings the P and S fields of its tile plus a 2N halo into shared
//      memory by tensor copies (cp.async.bulk.tensor boxes completing on an
//      mbarrier, bounded wait) and sums them to the total displacement U;
//   2. computes the S-stage (theta, omega and the four Q fields, with the
//      S-stage CPML memory) for its tile plus an N halo, keeping it on chip:
//      halo cells are recomputed by both neighbouring CTAs, so the six
//      intermediate fields never reach HBM;
//   3. computes the U-stage for its own cells: eight staggered derivatives of
//      the S fields, the U-stage CPML memory, the P/S leapfrog, and writes the
//      new level over the oldest one (ping-pong of the P/S pairs makes the halo
//      reads of phase 1 race-free).
// Receiver extraction, record injection, boundary-strip save/restore and the
// zero-lag imaging condition ride along in the same launch.
//
// Cost structure.  Tiles whose whole neighbourhood lies inside the update
// domain, away from the boundary ring, the source and the receiver row are
// "clean" and run no per-cell test at all; the few "edge" tiles mask per
// float4.  Damping and edge handling are uniform run-time branches of a
// single code path: separate unrolled variants per tile class overflow the
// instruction cache.  Arithmetic is written with explicit roundings that reproduce the
// reference's compiled expressions exactly (established by probing the
// compiler's contractions on sm_100a):
//   derivative  acc = fma(a_1, d_1, a_2 d_2);  acc = fma(a_k, d_k, acc);  acc / h
//   CPML        fma(fma(d, e, -(d m)), dt, m)              (PS:281, PS:368)
//   leapfrog    fma(dt^2, s, fma(2, now, -past))           (PS:291-294)
//   imaging     acc + fma(p, q, u v)                       (PS:1434-1436)
// which lets x-derivatives and all per-cell updates run as packed f32x2
// instructions (two lanes of one float4 per instruction) without changing a
// single rounding.  Division by the spacing uses the Markstein correction
//   q0 = x r;  q = fma(fma(-q0, h, x), r, q0),   r = RN(1/h),
// which returns the correctly rounded quotient for every normal result
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990; checked exhaustively against
// IEEE division on sm_100a for the spacings in use); quotients near the
// subnormal range go through an exact scaled form (div_tiny below).
#pragma once
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ouc_internal.h"

namespace ouc {

template <int N>
struct TileGeo {
    static constexpr int TX = 32;                  // tile rows (x)
    static constexpr int TZ = 64;                  // tile columns (z)
    static constexpr int SHX = (N + 1) & ~1;       // S-stage row halo (even)
    static constexpr int HS = (N + 3) & ~3;        // S-stage column halo (float4 aligned)
    static constexpr int HU = (HS + N + 3) & ~3;   // U column halo
    static constexpr int NB = (N + 3) / 4;         // float4 blocks on each side of a z window
    static constexpr int UR = TX + 2 * (SHX + N);  // U rows held
    static constexpr int UC = TZ + 2 * HU;         // U columns held
    static constexpr int SR = TX + 2 * SHX;        // rows of theta/omega/Qxz/Qzz
    static constexpr int SC = TZ + 2 * HS;         // columns of theta/omega/Qxx/Qzx
    static constexpr int oUx = 0;
    static constexpr int oUz = oUx + UR * UC;
    static constexpr int oTh = oUz + UR * UC;
    static constexpr int oOm = oTh + SR * SC;
    static constexpr int oQxz = oOm + SR * SC;     // SR x TZ (x-derivative only)
    static constexpr int oQzz = oQxz + SR * TZ;
    static constexpr int oQxx = oQzz + SR * TZ;    // TX x SC (z-derivative only)
    static constexpr int oQzx = oQxx + TX * SC;
    static constexpr int floats = oQzx + TX * SC;
    static constexpr int bytes = floats * 4;
    static constexpr int itemsA = (SR / 4) * (TZ / 4);        // S items over all rows, own columns
    static constexpr int itemsB = (TX / 4) * (2 * HS / 4);    // S items over own rows, halo columns
    static_assert(SR % 4 == 0, "S rows must group by 4");
    static_assert(itemsA + itemsB <= kThreads, "one S item per thread");
    static_assert((TX / 2) * (TZ / 4) == kThreads, "one U item per thread");
};

// ---- small helpers -----------------------------------------------------------
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float4 cat4(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float comp(const float4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(float4& v, int k, float x) {
    if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b with one rounding: fma(b, -1, a)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return cat4(add2(lo2(a), lo2(b)), add2(hi2(a), hi2(b))); }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) { return cat4(sub2(lo2(a), lo2(b)), sub2(hi2(a), hi2(b))); }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) { return cat4(mul2(lo2(a), lo2(b)), mul2(hi2(a), hi2(b))); }
__device__ __forceinline__ float4 mul4s(float4 a, float s) { return cat4(mul2(lo2(a), dup2(s)), mul2(hi2(a), dup2(s))); }
// Field accesses of phases 2 and 3 in the global space (ld/st.global.cg,
// cached in L2 only): unlike accesses through generic pointers, the
// compiler may order them freely against the shared-memory accesses
// (-1 to -3 % per launch measured).
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void stg4(float* p, float4 v) { __stcg(reinterpret_cast<float4*>(p), v); }
__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }

struct Div {
    float h, r;    // spacing and RN(1/h)
    unsigned tb;   // 2 bits(T) - 1: dividends with 0 < |x| < T take div_tiny
};
// T bounds every dividend whose quotient estimate RN(x r) lies below 2^-124:
// such an x has |x| < 2^-124 / r <= 2^-124 h (1 + 2^-23) (r = RN(1/h)), so
// T = 2^-124 h (1 + 2^-22), each product rounded up.
__device__ __forceinline__ Div make_div(float h, float r) {
    const float t = __fmul_ru(__fmul_ru(h, 1.0f + 0x1p-22f), 0x1p-124f);
    return Div{h, r, __float_as_uint(t) * 2u - 1u};
}

// Quotients below 2^-124 (the subnormal neighbourhood, common in the band of
// tiny values that runs ahead of a wavefront) cannot take the Markstein form,
// whose remainder would leave the normal range.  The guard tests the
// dividend (0 < |x| < T, Div::tb), a superset of the dividends whose quotient
// estimate lies below 2^-124, and div_tiny divides those exactly in single
// precision: the dividend scaled by 2^64 (exact) has a normal quotient, which
// the Markstein form rounds correctly; scaled back by 2^-64 it is exact when
// normal, and a subnormal result is the scaled quotient rounded to the
// subnormal grid -- which can differ from the correctly rounded x / h only
// when the scaled quotient lies exactly half-way between two subnormals, a
// tie that the sign of the exact remainder a - q h settles.  Equal to IEEE
// division for every tiny dividend (exhaustive checks on the CPU and on
// sm_100a for the spacings in use), and much cheaper than the double-
// precision division it replaces (13 % of the whole RTM step at c2).
__device__ __forceinline__ float div_tiny(float x, float h, float r) {
    const float a = __fmul_rn(fabsf(x), 0x1p64f);   // exact: |x| >= 2^-149
    const float q0 = __fmul_rn(a, r);
    const float qa = __fmaf_rn(__fmaf_rn(-q0, h, a), r, q0);   // RN(a / h), a normal number
    float q;
    if (qa >= 0x1p-62f) {
        q = __fmul_rn(qa, 0x1p-64f);                 // normal result: the scaling is exact
    } else {
        const float t = __fmul_rn(qa, 0x1p85f);      // the result in units of 2^-149, below 2^23
        const float ra = __fmaf_rn(-qa, h, a);       // exact remainder
        const float ft = truncf(t);
        float n = rintf(t);
        if (__fsub_rn(t, ft) == 0.5f) n = ra > 0.f ? __fadd_rn(ft, 1.f) : (ra < 0.f ? ft : n);
        q = __int_as_float((int)n);                  // n x 2^-149
    }
    return copysignf(q, x);
}
__device__ __forceinline__ float4 div4(float4 x, const Div& d) {
    const float2 q0l = mul2(lo2(x), dup2(d.r)), q0h = mul2(hi2(x), dup2(d.r));
    float4 q = cat4(fma2(fma2(q0l, dup2(-d.h), lo2(x)), dup2(d.r), q0l),
                    fma2(fma2(q0h, dup2(-d.h), hi2(x)), dup2(d.r), q0h));
    // 0 < |x| < T, on the bits: 2 bits(x) - 1 drops the sign and wraps a zero to the largest value
    const bool tiny = (__float_as_uint(x.x) * 2u - 1u < d.tb) | (__float_as_uint(x.y) * 2u - 1u < d.tb) |
                      (__float_as_uint(x.z) * 2u - 1u < d.tb) | (__float_as_uint(x.w) * 2u - 1u < d.tb);
    if (tiny)
        q = make_float4(div_tiny(x.x, d.h, d.r), div_tiny(x.y, d.h, d.r), div_tiny(x.z, d.h, d.r),
                        div_tiny(x.w, d.h, d.r));
    return q;
}
// CPML memory update fma(fma(d, e, -(d m)), dt, m), packed
__device__ __forceinline__ float2 cpml2(float2 m, float2 d, float2 e, float dt) {
    const float2 dm = mul2(d, m);
    return fma2(fma2(d, e, make_float2(-dm.x, -dm.y)), dup2(dt), m);
}
__device__ __forceinline__ float4 cpml4(float4 m, float4 d, float4 e, float dt) {
    return cat4(cpml2(lo2(m), lo2(d), lo2(e), dt), cpml2(hi2(m), hi2(d), hi2(e), dt));
}

// Staggered derivative of four consecutive z cells starting at `row`
// (16-byte aligned shared-memory pointer at the first of the four cells).
// PLUS: sum_k a_k (f[j+k] - f[j-k+1]);  MINUS: sum_k a_k (f[j+k-1] - f[j-k]).
// Scalar: the z-shifted pairs do not sit in aligned register pairs.
template <int N, bool PLUS>
__device__ __forceinline__ float4 dz4(const float* row, const float* a, const Div& dv) {
    constexpr int NB = (N + 3) / 4;
    float w[4 * (2 * NB + 1)];
#pragma unroll
    for (int b = 0; b < 2 * NB + 1; ++b) {
        const float4 v = ld4(row + 4 * (b - NB));
        w[4 * b + 0] = v.x; w[4 * b + 1] = v.y; w[4 * b + 2] = v.z; w[4 * b + 3] = v.w;
    }
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int c = 4 * NB + q;
        // fma(a_1, d_1, a_2 d_2), then fma(a_k, d_k, acc)
        const float d0 = PLUS ? __fsub_rn(w[c + 1], w[c]) : __fsub_rn(w[c], w[c - 1]);
        const float d1 = PLUS ? __fsub_rn(w[c + 2], w[c - 1]) : __fsub_rn(w[c + 1], w[c - 2]);
        float acc = __fmaf_rn(a[0], d0, __fmul_rn(a[1], d1));
#pragma unroll
        for (int k = 2; k < N; ++k)
            acc = PLUS ? __fmaf_rn(a[k], __fsub_rn(w[c + k + 1], w[c - k]), acc)
                       : __fmaf_rn(a[k], __fsub_rn(w[c + k], w[c - k - 1]), acc);
        o[q] = acc;
    }
    return div4(make_float4(o[0], o[1], o[2], o[3]), dv);
}

// Staggered x derivatives of RR consecutive rows of one float4 column,
// packed two lanes per instruction.  `col` points at row r0 of the column in
// shared memory, `st` is the row stride in floats; window rows r0-N ..
// r0+RR-1+N are read once.
template <int N, int RR, bool PLUS>
__device__ __forceinline__ void dx4(const float* col, int st, const float* a, const Div& dv, float4 (&out)[RR]) {
    float4 w[RR + 2 * N];
#pragma unroll
    for (int k = 0; k < RR + 2 * N; ++k) {
        if (PLUS ? k >= 1 : k < RR + 2 * N - 1) w[k] = ld4(col + (k - N) * st);
    }
#pragma unroll
    for (int q = 0; q < RR; ++q) {
        const int c = q + N;
        float2 acl, ach;
        {   // fma(a_1, d_1, a_2 d_2)
            const int hi0 = PLUS ? c + 1 : c, lo0 = PLUS ? c : c - 1;
            const int hi1 = PLUS ? c + 2 : c + 1, lo1 = PLUS ? c - 1 : c - 2;
            acl = fma2(dup2(a[0]), sub2(lo2(w[hi0]), lo2(w[lo0])), mul2(dup2(a[1]), sub2(lo2(w[hi1]), lo2(w[lo1]))));
            ach = fma2(dup2(a[0]), sub2(hi2(w[hi0]), hi2(w[lo0])), mul2(dup2(a[1]), sub2(hi2(w[hi1]), hi2(w[lo1]))));
        }
#pragma unroll
        for (int k = 2; k < N; ++k) {
            const int hi = PLUS ? c + k + 1 : c + k, lo = PLUS ? c - k : c - k - 1;
            acl = fma2(dup2(a[k]), sub2(lo2(w[hi]), lo2(w[lo])), acl);
            ach = fma2(dup2(a[k]), sub2(hi2(w[hi]), hi2(w[lo])), ach);
        }
        out[q] = div4(cat4(acl, ach), dv);
    }
}

// ---- bulk asynchronous copies and mbarriers ----------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// One hardware-suspended wait on phase `parity`: the thread sleeps until the
// phase completes or a time limit of about 0.1 ms passes (no busy polling).
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity), "r"(100000u)
        : "memory");
    return ok != 0;
}
// Bounded wait on phase `parity`: false after about 200 suspended tries
// (some 20 ms; a tile's copies take microseconds).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
    for (int k = 0; k < 200; ++k)
        if (mbar_try(b, parity)) return true;
    return false;
}
// One box of a 4-D tensor map (tile mode, no multicast) into shared memory
// at `dst` (128-byte aligned), completing its bytes on the mbarrier.  The
// innermost coordinate c0 must be a multiple of 4 (16 bytes of floats).
__device__ __forceinline__ void tma_box4(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(b))
        : "memory");
}
// L2 prefetch of one box of a 4-D tensor map (no shared-memory write, no
// completion to wait for).  Same coordinate rule as tma_box4.
__device__ __forceinline__ void tma_prefetch_box4(const CUtensorMap* map, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Per-launch, per-shot constants.
struct ShotView {
    int b;                 // shot of the batch
    int sx, sz, rz, src_type;
    const float* wavelet;
    float* rec_x;          // gather row t (kFwd) or nullptr
    float* rec_z;
    const float* inj_x;    // gather row t (kRcv)
    const float* inj_z;
    bool strips;           // the shot has boundary strips
    size_t off;            // state offset of this shot (floats)
};

// Per-shot grid geometry read from the shot descriptor.
struct Geo {
    int X;
    Ring ring;
    const float* vp2;
    const float* vs2;
    const float* ax;
    const float* az;
    const float* bx;
    const float* bz;
};

__device__ __forceinline__ Geo geo_of(const ShotDesc& d) {
    Geo gm;
    gm.X = d.X; gm.ring = d.ring; gm.vp2 = d.vp2; gm.vs2 = d.vs2; gm.ax = d.ax; gm.az = d.az;
    gm.bx = d.bx; gm.bz = d.bz;
    return gm;
}

__device__ __forceinline__ ShotView shot_view(const StepArgs& p, int b) {
    const ShotDesc& d = p.shots[b];
    ShotView v;
    v.b = b;
    v.sx = d.sx; v.sz = d.sz; v.rz = d.rz; v.src_type = d.src_type;
    v.wavelet = d.wavelet;
    v.rec_x = p.record ? d.gather_x + (size_t)p.t * d.X : nullptr;
    v.rec_z = p.record ? d.gather_z + (size_t)p.t * d.X : nullptr;
    v.inj_x = d.gather_x + (size_t)p.t * d.X;
    v.inj_z = d.gather_z + (size_t)p.t * d.X;
    v.strips = d.strips != nullptr;
    v.off = d.off;
    return v;
}

// ---- boundary-strip elements (StripPrec) -----------------------------------
// Strip pointers are formed inside the ring passes from the shot descriptor,
// so that they hold no registers through the rest of the step.

// 2^k for k in [-126, 127]
__device__ __forceinline__ float pow2f(int k) { return __int_as_float((k + 127) << 23); }

// v * 2^k for k in [-252, 254], as two exact power-of-two multiplies
__device__ __forceinline__ float scale2(float v, int k) {
    const int k1 = k / 2;
    return v * pow2f(k1) * pow2f(k - k1);
}

// kStripF16 scale exponent of a slot/field whose largest |v| has the bits
// `a` (a non-negative float): that value maps into [2^14, 2^15), so every
// scaled value is below 2^15 and converts to a finite half.
__device__ __forceinline__ int f16_exp(unsigned a) {
    if (a == 0) return 0;
    const int e = (a >> 23) ? (int)(a >> 23) - 127 : (31 - __clz(a)) - 149;   // floor(log2 a)
    return 14 - e;
}

__device__ __forceinline__ size_t slot_bytes(const StepArgs& p, const ShotDesc& d) {
    return d.strip_slot * (size_t)strip_elem_bytes(p.strip_prec);
}

// Slot `slot` of a shot's strips (element type per p.strip_prec).
__device__ __forceinline__ const void* strip_slot_ptr(const StepArgs& p, const ShotDesc& d, int slot) {
    return static_cast<const char*>(d.strips) + (size_t)slot * slot_bytes(p, d);
}

__device__ __forceinline__ float strip_get(const StepArgs& p, const void* base, const unsigned* amax, int f, int idx) {
    if (p.strip_prec == kStripF32) return static_cast<const float*>(base)[idx];
    if (p.strip_prec == kStripBF16) return __bfloat162float(static_cast<const __nv_bfloat16*>(base)[idx]);
    return scale2(__half2float(static_cast<const __half*>(base)[idx]), -f16_exp(amax[f]));
}

// Where the forward step writes slot t: the strips themselves (f32, bf16) or
// the f16 staging ring slot t & 1 (floats).
__device__ __forceinline__ void* strip_save_ptr(const StepArgs& p, const ShotDesc& d) {
    if (p.strip_prec == kStripF16) return d.stage + (size_t)(p.t & 1) * d.strip_slot;
    return static_cast<char*>(d.strips) + (size_t)p.t * slot_bytes(p, d);
}

__device__ __forceinline__ void strip_put(const StepArgs& p, void* base, int idx, float v) {
    if (p.strip_prec == kStripBF16) static_cast<__nv_bfloat16*>(base)[idx] = __float2bfloat16_rn(v);
    else static_cast<float*>(base)[idx] = v;
}

// Fold per-thread maxima of |v| into a slot's field maxima (f16 strips):
// one atomic per warp and field.
template <int NF>
__device__ __forceinline__ void amax_commit(unsigned* amax, int f0, const float (&m)[NF]) {
#pragma unroll
    for (int q = 0; q < NF; ++q) {
        float v = m[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0 && v > 0.f) atomicMax(amax + f0 + q, __float_as_uint(v));
    }
}

// Tile flags, uniform per CTA.
struct TileFlags {
    bool px, pz;    // the S region touches the x / z damping layers
    bool border;    // some S-region or own cell lies outside the update domain
    bool ring;      // boundary-ring work: strip save (forward) or restore (reconstruction)
    bool src;       // the source cell lies in the S region (own cells for a force source)
    bool inj;       // the receiver row crosses the U box (receiver mode)
};

__device__ __forceinline__ bool rect_meets_ring(const Ring& R, int i0, int i1, int j0, int j1) {
    const int L = R.L, N = R.N, X = R.X, Z = R.Z;
    const bool meets_box = i0 < X - L + N && i1 > L - N && j0 < Z - L + N && j1 > L - N;
    const bool inside_deep = i0 >= L + N && i1 <= X - L - N && j0 >= L + N && j1 <= Z - L - N;
    return meets_box && !inside_deep;
}

// Visit, cooperatively over the CTA, the boundary-ring cells inside the
// rectangle [i0, i1) x [j0, j1) (global coordinates): f(i, j, ring index).
// The four bands are rectangles, so each visit is a plain 2-D loop and the
// strip accesses are contiguous along z.
template <class F>
__device__ __forceinline__ void for_ring(const Ring& R, int i0, int i1, int j0, int j1, F&& f) {
    const int L = R.L, N = R.N, X = R.X, Z = R.Z, n2 = 2 * N, W = R.W, hm = R.H - 4 * N;
#pragma unroll 1
    for (int b = 0; b < 4; ++b) {
        int bi0, bi1, bj0, bj1, base, stride;
        if (b == 0) { bi0 = L - N; bi1 = X - L + N; bj0 = L - N; bj1 = L + N; base = 0; stride = n2; }
        else if (b == 1) { bi0 = L - N; bi1 = X - L + N; bj0 = Z - L - N; bj1 = Z - L + N; base = W * n2; stride = n2; }
        else if (b == 2) { bi0 = L - N; bi1 = L + N; bj0 = L + N; bj1 = Z - L - N; base = 2 * W * n2; stride = hm; }
        else { bi0 = X - L - N; bi1 = X - L + N; bj0 = L + N; bj1 = Z - L - N; base = 2 * W * n2 + n2 * hm; stride = hm; }
        const int ia = max(i0, bi0), ib = min(i1, bi1), ja = max(j0, bj0), jb = min(j1, bj1);
        if (ia >= ib || ja >= jb) continue;
        const int w = jb - ja, n = (ib - ia) * w;
        // k / w as a multiply-high by m = ceil(2^32 / w): exact for k < 2^16
        // and w <= 2^16 (the error k (m - 2^32 / w) / 2^32 < 2^-16 stays
        // below 1/w); the rectangles here hold well under 2^16 cells
        const unsigned m = w > 1 ? 0xFFFFFFFFu / (unsigned)w + 1u : 0u;
        for (int k = threadIdx.x; k < n; k += kThreads) {
            const int q = w > 1 ? (int)__umulhi((unsigned)k, m) : k;
            const int i = ia + q, j = ja + (k - q * w);
            f(i, j, base + (i - bi0) * stride + (j - bj0));
        }
    }
}

template <int N, int MODE>
__device__ __forceinline__ TileFlags tile_flags(const StepArgs& p, const Geo& gm, const ShotView& sv, int x0, int z0) {
    using G = TileGeo<N>;
    const int X = gm.X, Z = p.Z, L = p.L;
    TileFlags f;
    f.px = f.pz = false;
    f.ring = f.src = f.inj = false;
    const int s_i0 = x0 - G::SHX, s_i1 = x0 + G::TX + G::SHX, s_j0 = z0 - G::HS, s_j1 = z0 + G::TZ + G::HS;
    const bool src_in_s = sv.sx >= s_i0 && sv.sx < s_i1 && sv.sz >= s_j0 && sv.sz < s_j1;
    if (MODE == kRec) {
        f.border = !(x0 >= L && x0 + G::TX <= X - L && z0 >= L && z0 + G::TZ <= Z - L);
        f.ring = sv.strips &&
                 rect_meets_ring(gm.ring, x0 - G::SHX - N, x0 + G::TX + G::SHX + N, z0 - G::HU, z0 + G::TZ + G::HU);
        f.src = p.src_recon && src_in_s;
        return f;
    }
    // damping is non-zero for i < L or i > X-L (PS:2072-2080)
    f.px = s_i0 < L || s_i1 - 1 >= X - L;
    f.pz = s_j0 < L || s_j1 - 1 >= Z - L;
    f.border = !(s_i0 >= N && s_i1 <= X - N && s_j0 >= N && s_j1 <= Z - N);
    if (MODE == kFwd) {
        f.ring = p.save && sv.strips && rect_meets_ring(gm.ring, x0, x0 + G::TX, z0, z0 + G::TZ);
        f.src = (sv.src_type == 0 && src_in_s) ||
                (sv.src_type == 1 && sv.sx >= x0 && sv.sx < x0 + G::TX && sv.sz >= z0 && sv.sz < z0 + G::TZ);
    }
    if (MODE == kRcv) {
        f.inj = sv.rz >= z0 - G::HU && sv.rz < z0 + G::TZ + G::HU && x0 - G::SHX - N < X - L &&
                x0 + G::TX + G::SHX + N > L;
    }
    return f;
}

// L2 prefetch of the strip elements that a reconstruction tile restores:
// the ring cells of its U box (slot_u: Ux, Uz) and of its S region (slot_s:
// theta, omega and the four Q fields), over the same band rectangles as
// for_ring.  The strips were written during the forward pass and come from
// DRAM; prefetched at the tile's start, their latency runs under the U-box
// copy and the S-stage instead of stalling the restore loops.  One 128-byte
// line per prefetch, at element addresses inside the strip slots.
template <int N>
__device__ __forceinline__ void prefetch_ring(const StepArgs& p, const Geo& gm, const ShotDesc& d, int x0, int z0) {
    using G = TileGeo<N>;
    const Ring& R = gm.ring;
    const int L = R.L, X = R.X, Z = R.Z, n2 = 2 * R.N, W = R.W, hm = R.H - 4 * R.N;
    const int eb = strip_elem_bytes(p.strip_prec), per_line = 128 / eb;
#pragma unroll 1
    for (int part = 0; part < 2; ++part) {
        const int i0 = part ? x0 - G::SHX : x0 - G::SHX - N, i1 = part ? x0 + G::TX + G::SHX : x0 - G::SHX - N + G::UR;
        const int j0 = part ? z0 - G::HS : z0 - G::HU, j1 = part ? z0 + G::TZ + G::HS : z0 - G::HU + G::UC;
        const char* slot = static_cast<const char*>(strip_slot_ptr(p, d, part ? p.slot_s : p.slot_u));
        const int f0 = part ? (int)kSTh : (int)kSUx, nf = part ? 6 : 2;
#pragma unroll 1
        for (int b = 0; b < 4; ++b) {
            int bi0, bi1, bj0, bj1, base, stride;
            if (b == 0) { bi0 = L - R.N; bi1 = X - L + R.N; bj0 = L - R.N; bj1 = L + R.N; base = 0; stride = n2; }
            else if (b == 1) { bi0 = L - R.N; bi1 = X - L + R.N; bj0 = Z - L - R.N; bj1 = Z - L + R.N; base = W * n2; stride = n2; }
            else if (b == 2) { bi0 = L - R.N; bi1 = L + R.N; bj0 = L + R.N; bj1 = Z - L - R.N; base = 2 * W * n2; stride = hm; }
            else { bi0 = X - L - R.N; bi1 = X - L + R.N; bj0 = L + R.N; bj1 = Z - L - R.N; base = 2 * W * n2 + n2 * hm; stride = hm; }
            const int ia = max(i0, bi0), ib = min(i1, bi1), ja = max(j0, bj0), jb = min(j1, bj1);
            if (ia >= ib || ja >= jb) continue;
            const int rows = ib - ia, nl = (jb - ja + per_line - 1) / per_line;   // lines of one row's run
            // row-major (field, row, line) index decoded by multiply-high, as in for_ring
            const int per_f = rows * nl;
            const unsigned mf = per_f > 1 ? 0xFFFFFFFFu / (unsigned)per_f + 1u : 0u;
            const unsigned ml = nl > 1 ? 0xFFFFFFFFu / (unsigned)nl + 1u : 0u;
            for (int k = threadIdx.x; k < nf * per_f; k += kThreads) {
                const int f = per_f > 1 ? (int)__umulhi((unsigned)k, mf) : k, rem = k - f * per_f;
                const int row = nl > 1 ? (int)__umulhi((unsigned)rem, ml) : rem, l = rem - row * nl;
                // element of the run: l * per_line < jb - ja
                const int e = base + (ia + row - bi0) * stride + (ja - bj0) + l * per_line;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(slot + ((size_t)(f0 + f) * R.R + e) * eb));
            }
        }
    }
}

template <int N, int MODE>
__device__ __forceinline__ bool u_live(const StepArgs& p, const Geo& gm, int gi, int gj) {
    if (MODE == kRec) return gi >= p.L && gi < gm.X - p.L && gj >= p.L && gj < p.Z - p.L;
    return gi >= N && gi < gm.X - N && gj >= N && gj < p.Z - N;
}

// L2 prefetch of a tile's thread-loaded operands, so that the loads of
// phases 2 and 3 find their lines in flight or resident: the oldest level
// (read and overwritten in phase 3) and, for the reconstruction, the
// receiver level and the imaging accumulators over the own cells -- one
// tensor prefetch per field (the state block's own-cell map) -- and the
// model over the S region (phase 2), one 128-byte line per instruction
// (every address inside the field allocations, guard rows and columns
// included).  The U box of phase 1 arrives by tensor copies.
template <int N, int MODE>
__device__ __forceinline__ void prefetch_tile(const StepArgs& p, const Geo& gm, int x0, int z0, int slot,
                                              const TileFlags& fl) {
    using G = TileGeo<N>;
    constexpr int TX = G::TX, TZ = G::TZ, SHX = G::SHX, HS = G::HS;
    const int tid = threadIdx.x;
    const int P = p.pitch;
    // own cells of the oldest level (and, reconstructing, of the receiver
    // level and the accumulators): one tensor prefetch per field
    if (tid == 32) {
        const int c0 = z0 + kZOFF, c1 = x0 + kGX;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (p.past_field[f] >= 0) tma_prefetch_box4(&p.own_map, c0, c1, p.past_field[f], slot);
            if (MODE == kRec && p.rcv_field[f] >= 0) tma_prefetch_box4(&p.own_map, c0, c1, p.rcv_field[f], slot);
            if (MODE == kRec && f < 3 && p.acc_field[f] >= 0)
                tma_prefetch_box4(&p.own_map, c0, c1, p.acc_field[f], slot);
        }
    }
    // in tiles that meet the damping layers: the S-stage CPML memories over
    // the S region and the U-stage ones over the own cells, the fields that
    // the tile's layers (x, z) use
    if (MODE != kRec && tid == 64 && (fl.px || fl.pz)) {
        const int s0 = z0 - HS + kZOFF, s1 = x0 - SHX + kGX, c0 = z0 + kZOFF, c1 = x0 + kGX;
        // S-stage: x layers xx (0) and zx (3), z layers zz (1) and xz (2)
#pragma unroll
        for (int f = 0; f < 4; ++f)
            if (((f == 0 || f == 3) ? fl.px : fl.pz) && p.fold_field[f] >= 0)
                tma_prefetch_box4(&p.s_map, s0, s1, p.fold_field[f], slot);
        // U-stage: z layers C A Tz Wz (0 3 5 6), x layers E B Tx Wx (1 2 4 7)
#pragma unroll
        for (int f = 0; f < 8; ++f)
            if (((f == 0 || f == 3 || f == 5 || f == 6) ? fl.pz : fl.px) && p.o_field[f] >= 0)
                tma_prefetch_box4(&p.own_map, c0, c1, p.o_field[f], slot);
    }
    // the model over the S region: Vp^2, Vs^2 and, in damping tiles, the
    // damping profiles of the tile's layers
    constexpr int kSPer = (TZ + 2 * HS + 31) / 32 + 1;
    constexpr int kSLines = (TX + 2 * SHX) * kSPer;
    const int nm = MODE == kRec ? 2 : 2 + (fl.px ? 1 : 0) + (fl.pz ? 1 : 0);
    for (int k = tid; k < nm * kSLines; k += kThreads) {
        const int f = k / kSLines, l = k - f * kSLines;
        const int g = (x0 - SHX + l / kSPer) * P + (z0 - HS) + 32 * (l % kSPer);
        const float* m = f == 0 ? gm.vp2 : f == 1 ? gm.vs2 : (f == 2 && fl.px) ? gm.ax : gm.az;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(m + g));
    }
}

// Issue the four tensor copies of a tile's U box (one thread): the UC x UR
// box of each P/S field of the current level, completing on the CTA's
// mbarrier -- P into the U arrays, S into the S-stage area, which is unused
// until phase 2.  The whole 83 KB box is in flight at once and no thread
// holds it in registers.  Called as early as the tile is known, so that the
// copies overlap the tile's set-up.  `slot` is the shot's index in the
// launch, which is its slot in the state block (its fields lie slot x
// shot_stride floats after shot 0's).
template <int N>
__device__ __forceinline__ void issue_u_box(const StepArgs& p, float* sm, int x0, int z0, int slot, uint64_t* bar) {
    using G = TileGeo<N>;
    static_assert(G::floats - G::oTh >= 2 * G::UR * G::UC, "S staging fits the S-stage area");
    static_assert((G::oUz * 4) % 128 == 0 && (G::oTh * 4) % 128 == 0 && (G::UR * G::UC * 4) % 128 == 0,
                  "tensor-copy destinations are 128-byte aligned");
    mbar_arrive_tx(bar, 4u * G::UR * G::UC * 4u + p.copy_tx_extra);
    // a previous tile's shared-memory accesses (generic proxy) precede these writes
    fence_proxy_async();
    // allocation coordinates: column z0 - HU + kZOFF (a multiple of 4), row x0 - SHX - N + kGX (>= 0)
    const int c0 = z0 - G::HU + kZOFF, c1 = x0 - G::SHX - N + kGX;
    float* stS = sm + G::oTh;
    tma_box4(sm + G::oUx, &p.box_map, c0, c1, p.now_field[0], slot, bar);
    tma_box4(sm + G::oUz, &p.box_map, c0, c1, p.now_field[1], slot, bar);
    tma_box4(stS, &p.box_map, c0, c1, p.now_field[2], slot, bar);
    tma_box4(stS + G::UR * G::UC, &p.box_map, c0, c1, p.now_field[3], slot, bar);
}

// Offsets within one field are 32-bit ints (row * pitch + column, guard rows
// negative): ouc_create refuses grids whose field allocation exceeds 2^31
// floats, and the 32-bit multiply-adds are fewer instructions than the
// 64-bit ones (+1.3 % measured).
// One tile's step, after issue_u_box.  `bar` is the CTA's mbarrier
// (initialised, count 1) and `parity` the phase that this tile's copies
// complete.  Returns false, with
// bit 0 of *p.err set, when the copies did not land within the wait's bound
// (or an earlier launch had recorded such a failure): the tile is then left
// unwritten and the host reports OUC_ETIMEOUT after the call.
template <int N, int MODE>
__device__ __forceinline__ bool step_tile(const StepArgs& p, const Geo& gm, const ShotView& sv, float* sm, int x0, int z0,
                                          const TileFlags& f, uint64_t* bar, unsigned parity) {
    using G = TileGeo<N>;
    constexpr int TX = G::TX, TZ = G::TZ, SHX = G::SHX, HS = G::HS, HU = G::HU, UC = G::UC, SC = G::SC;
    const int tid = threadIdx.x;
    const int P = p.pitch;
    const size_t R = gm.ring.R;
    float* sUx = sm + G::oUx;
    float* sUz = sm + G::oUz;
    float* sTh = sm + G::oTh;
    float* sOm = sm + G::oOm;
    float* sQxz = sm + G::oQxz;
    float* sQzz = sm + G::oQzz;
    float* sQxx = sm + G::oQxx;
    float* sQzx = sm + G::oQzx;
    float a[N];
#pragma unroll
    for (int k = 0; k < N; ++k) a[k] = p.a[k];
    const Div dvx = make_div(p.dx, p.rdx), dvz = make_div(p.dz, p.rdz);
    const size_t off = sv.off;
    const float* nowp[4] = {p.now[0] + off, p.now[1] + off, p.now[2] + off, p.now[3] + off};
    const int ux_i0 = x0 - SHX - N, ux_j0 = z0 - HU;   // global origin of the U box

    // ---- phase 1: U = P + S over the tile and a 2N halo ---------------------
    // The box's four tensor copies were issued at the start of the tile
    // (issue_u_box); wait for them, then one shared-memory pass adds S to P.
    float* stS = sm + G::oTh;   // Sx then Sz staging, UR x UC each
    const int err_word = p.err ? *(volatile const int*)p.err : 0;   // consumed after the wait
    const bool landed = mbar_wait(bar, parity);
    if (!__syncthreads_and(landed && !(err_word & 1))) {
        // a failed wait: one more bounded wait lets copies in flight land
        // before the shared memory is reused or released; then report
        if (tid == 0) {
            if (!landed) mbar_wait(bar, parity);
            if (p.err) atomicOr(p.err, 1);
        }
        __syncthreads();
        return false;
    }
    for (int idx = tid; idx < G::UR * (UC / 4); idx += kThreads) {
        st4(sUx + 4 * idx, add4(ld4(sUx + 4 * idx), ld4(stS + 4 * idx)));                  // Ux = Px + Sx (PS:302)
        st4(sUz + 4 * idx, add4(ld4(sUz + 4 * idx), ld4(stS + G::UR * UC + 4 * idx)));     // Uz = Pz + Sz
    }
    if (MODE == kRcv && f.inj) {
        __syncthreads();
        // load_record (PS:1471-1483): the receiver row is overwritten by the
        // record over the interior x range before the S-stage reads it
        const int col = sv.rz - ux_j0;
        for (int r = tid; r < G::UR; r += kThreads) {
            const int gi = ux_i0 + r;
            if (gi >= p.L && gi < gm.X - p.L) {
                sUx[r * UC + col] = sv.inj_x[gi];
                sUz[r * UC + col] = sv.inj_z[gi];
            }
        }
    }
    if (MODE == kRec && f.ring) {
        __syncthreads();
        // reconstruction: the ring comes from the saved strips (read_wavefiled1, PS:1344-1376)
        const ShotDesc& d = p.shots[sv.b];
        const void* su = strip_slot_ptr(p, d, p.slot_u);
        const unsigned* am = d.amax ? d.amax + (size_t)p.slot_u * kStripFields : nullptr;
        // both loads before the stores: a shared store through a generic
        // pointer would otherwise order the second load behind the first
        // load's round trip
        for_ring(gm.ring, ux_i0, ux_i0 + G::UR, ux_j0, ux_j0 + UC, [&](int i, int j, int ri) {
            const int o = (i - ux_i0) * UC + (j - ux_j0);
            const float ux = strip_get(p, su, am, kSUx, kSUx * R + ri);
            const float uz = strip_get(p, su, am, kSUz, kSUz * R + ri);
            sUx[o] = ux;
            sUz[o] = uz;
        });
    }
    __syncthreads();

    // ---- phase 2: S-stage on the tile plus an N halo -------------------------
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
        const bool ownc = c >= 0 && c < TZ;
        // rows of the x-derivative window per iteration: 2 (measured 1.8 %
        // faster than 4 at c2, batch 16: less code in the hot loop)
        constexpr int P2R = 2;
#pragma unroll 1
        for (int q0 = 0; q0 < 4; q0 += P2R) {
        // the model's operands first: their latency runs under the derivatives
        float4 vp2r[P2R], vs2r[P2R];
#pragma unroll
        for (int qq = 0; qq < P2R; ++qq) {
            const int g = (x0 + r0 + q0 + qq) * P + (z0 + c);
            vp2r[qq] = ldg4(gm.vp2 + g);
            vs2r[qq] = ldg4(gm.vs2 + g);
        }
        float4 exx[P2R], ezx[P2R];
        dx4<N, P2R, false>(ux0 + q0 * UC, UC, a, dvx, exx);   // dvxdx = D-x Ux
        dx4<N, P2R, true>(uz0 + q0 * UC, UC, a, dvx, ezx);    // dvzdx = D+x Uz
#pragma unroll
        for (int qq = 0; qq < P2R; ++qq) {
            const int q = q0 + qq;
            const int r = r0 + q;
            const int gi = x0 + r;
            const int gjb = z0 + c;
            const float4 exz = dz4<N, true>(ux0 + q * UC, a, dvz);    // dvxdz = D+z Ux
            const float4 ezz = dz4<N, false>(uz0 + q * UC, a, dvz);   // dvzdz = D-z Uz
            const int g = gi * P + gjb;
            const float4 vp2 = vp2r[qq], vs2 = vs2r[qq];
            const bool own = ownc && r >= 0 && r < TX;
            float4 fxx = zero4(), fzz = zero4(), fxz = zero4(), fzx = zero4();
            if (f.px) {
                const float4 axv = ldg4(gm.ax + g);
                fxx = cpml4(ldg4(p.f_old[0] + off + g), axv, exx[qq], p.dt);
                fzx = cpml4(ldg4(p.f_old[3] + off + g), axv, ezx[qq], p.dt);
            }
            if (f.pz) {
                const float4 azv = ldg4(gm.az + g);
                fzz = cpml4(ldg4(p.f_old[1] + off + g), azv, ezz, p.dt);
                fxz = cpml4(ldg4(p.f_old[2] + off + g), azv, exz, p.dt);
            }
            // theta = Vp^2 (exx + ezz - Fxx - Fzz), omega = Vs^2 (exz - ezx - Fxz + Fzx) (PS:373-378);
            // outside the damping layers the memories are exact zeros and
            // adding or subtracting them leaves every rounding unchanged
            float4 th = mul4(vp2, sub4(sub4(add4(exx[qq], ezz), fxx), fzz));
            float4 om = mul4(vs2, add4(sub4(sub4(exz, ezx[qq]), fxz), fzx));
            float4 qzx = mul4(vs2, sub4(ezx[qq], fzx));
            float4 qzz = mul4(vs2, sub4(ezz, fzz));
            float4 qxz = mul4(vs2, sub4(exz, fxz));
            float4 qxx = mul4(vs2, sub4(exx[qq], fxx));
            if (MODE != kRec && f.border) {
                // cells outside [N, X-N) x [N, Z-N) are never updated by the
                // reference and stay zero
                const bool row_live = gi >= N && gi < gm.X - N;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int gj = gjb + k;
                    if (!(row_live && gj >= N && gj < p.Z - N)) {
                        set_comp(th, k, 0.f); set_comp(om, k, 0.f); set_comp(qzx, k, 0.f); set_comp(qzz, k, 0.f);
                        set_comp(qxx, k, 0.f); set_comp(qxz, k, 0.f);
                        set_comp(fxx, k, 0.f); set_comp(fzz, k, 0.f); set_comp(fxz, k, 0.f); set_comp(fzx, k, 0.f);
                    }
                }
            }
            if (own) {
                if (f.px) { stg4(p.f_new[0] + off + g, fxx); stg4(p.f_new[3] + off + g, fzx); }
                if (f.pz) { stg4(p.f_new[1] + off + g, fzz); stg4(p.f_new[2] + off + g, fxz); }
            }
            const int sr = r + SHX, scol = c + HS;
            st4(sTh + sr * SC + scol, th);
            st4(sOm + sr * SC + scol, om);
            if (groupA) {
                st4(sQxz + sr * TZ + c, qxz);
                st4(sQzz + sr * TZ + c, qzz);
            }
            if (r >= 0 && r < TX) {
                st4(sQxx + r * SC + scol, qxx);
                st4(sQzx + r * SC + scol, qzx);
            }
        }
        }
    }
    if (f.src && MODE != kRcv && !(MODE == kFwd && sv.src_type == 1)) {
        // source term on theta after the Q fields (PS:380); in the
        // reconstruction only where the level's theta is recomputed
        __syncthreads();
        if (tid == 0) {
            const int r = sv.sx - x0, c = sv.sz - z0;
            if ((r >= 0 && r < TX) || (c >= 0 && c < TZ)) {
                float* t = sTh + (r + SHX) * SC + (c + HS);
                *t = *t + sv.wavelet[MODE == kRec ? p.t + 1 : p.t];
            }
        }
    }
    if (f.ring) {
        __syncthreads();
        const ShotDesc& d = p.shots[sv.b];
        if (MODE == kRec) {
            // read_wavefiled2 (PS:1377-1424): theta, omega and the Q fields of the ring
            const void* ss = strip_slot_ptr(p, d, p.slot_s);
            const unsigned* am = d.amax ? d.amax + (size_t)p.slot_s * kStripFields : nullptr;
            // all six loads before any store (see the U restore above)
            for_ring(gm.ring, x0 - SHX, x0 + TX + SHX, z0 - HS, z0 + TZ + HS, [&](int i, int j, int ri) {
                const int r = i - x0, c = j - z0;
                const bool rin = r >= 0 && r < TX, cin = c >= 0 && c < TZ;
                float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (rin || cin) {
                    v[0] = strip_get(p, ss, am, kSTh, kSTh * R + ri);
                    v[1] = strip_get(p, ss, am, kSOm, kSOm * R + ri);
                }
                if (cin) {
                    v[2] = strip_get(p, ss, am, kSQxz, kSQxz * R + ri);
                    v[3] = strip_get(p, ss, am, kSQzz, kSQzz * R + ri);
                }
                if (rin) {
                    v[4] = strip_get(p, ss, am, kSQxx, kSQxx * R + ri);
                    v[5] = strip_get(p, ss, am, kSQzx, kSQzx * R + ri);
                }
                if (rin || cin) {
                    const int o = (r + SHX) * SC + (c + HS);
                    sTh[o] = v[0];
                    sOm[o] = v[1];
                }
                if (cin) {
                    sQxz[(r + SHX) * TZ + c] = v[2];
                    sQzz[(r + SHX) * TZ + c] = v[3];
                }
                if (rin) {
                    sQxx[r * SC + (c + HS)] = v[4];
                    sQzx[r * SC + (c + HS)] = v[5];
                }
            });
        }
        if (MODE == kFwd) {
            // save_wavefiled (PS:1230-1287): the S fields of the tile's ring cells
            void* s = strip_save_ptr(p, d);
            float m[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for_ring(gm.ring, x0, x0 + TX, z0, z0 + TZ, [&](int i, int j, int ri) {
                const int r = i - x0, c = j - z0;
                const int o = (r + SHX) * SC + (c + HS);
                const float v[6] = {sTh[o], sOm[o], sQzx[r * SC + (c + HS)], sQzz[(r + SHX) * TZ + c],
                                    sQxx[r * SC + (c + HS)], sQxz[(r + SHX) * TZ + c]};
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    strip_put(p, s, (kSTh + q) * R + ri, v[q]);
                    m[q] = fmaxf(m[q], fabsf(v[q]));
                }
            });
            if (p.strip_prec == kStripF16) amax_commit<6>(d.amax + (size_t)p.t * kStripFields, kSTh, m);
        }
    }
    __syncthreads();

    // ---- phase 3: U-stage on the tile's own cells (2 rows x 4 columns) ------
    {
        const int rr = 2 * (tid / (TZ / 4));
        const int c = 4 * (tid % (TZ / 4));
        const int scol = c + HS;
        const float dt = p.dt;
        // The x derivatives of a thread's two rows come from one window pass
        // (11 shared-memory loads per derivative instead of 20).  Where the
        // second row's values would stay in registers through the row loop
        // they cost spills, so the U box, free once the S-stage has read it,
        // holds them instead (one float4 per thread and value, stride
        // kThreads, conflict-free):
        //  - forward: tx, wx and dB of both rows above the first TX x TZ
        //    floats of the two U fields (those keep the new U for the strip
        //    pass); dE one row per pass;
        //  - receiver: all four of both rows from the start of the U fields;
        //  - reconstruction: the second row's values carried in registers;
        //  - U boxes too small for the above (N = 2): one row per pass.
        // Measured at c2, batch 16: forward -1.9 %, receiver -3.0 %,
        // reconstruction -2.0 % against one row per pass.
        constexpr bool kShare3 = MODE == kFwd && G::UR * G::UC >= TX * TZ + 12 * kThreads;
        constexpr bool kShare4 = MODE == kRcv && G::UR * G::UC >= 16 * kThreads;
        constexpr bool kCarry = MODE == kRec;
        float4* const c3x = reinterpret_cast<float4*>(sUx + TX * TZ) + tid;
        float4* const c3z = reinterpret_cast<float4*>(sUz + TX * TZ) + tid;
        float4* const c4x = reinterpret_cast<float4*>(sUx) + tid;
        float4* const c4z = reinterpret_cast<float4*>(sUz) + tid;
        float4 txr[2], wxr[2], dBr[2], dEr[2];
        if constexpr (kCarry || kShare3 || kShare4) {
            dx4<N, 2, true>(sTh + (rr + SHX) * SC + scol, SC, a, dvx, txr);    // dthetadx = D+x theta
            dx4<N, 2, false>(sOm + (rr + SHX) * SC + scol, SC, a, dvx, wxr);   // domegadx = D-x omega
            dx4<N, 2, false>(sQxz + (rr + SHX) * TZ + c, TZ, a, dvx, dBr);     // dux_zdx = D-x Qxz
        }
        if constexpr (kCarry || kShare4)
            dx4<N, 2, true>(sQzz + (rr + SHX) * TZ + c, TZ, a, dvx, dEr);      // duz_zdx = D+x Qzz
        if constexpr (kShare4) {
            c4x[0] = txr[0]; c4x[kThreads] = txr[1]; c4x[2 * kThreads] = wxr[0]; c4x[3 * kThreads] = wxr[1];
            c4z[0] = dBr[0]; c4z[kThreads] = dBr[1]; c4z[2 * kThreads] = dEr[0]; c4z[3 * kThreads] = dEr[1];
        }
        if constexpr (kShare3) {
            c3x[0] = txr[0]; c3x[kThreads] = txr[1]; c3x[2 * kThreads] = wxr[0];
            c3z[0] = wxr[1]; c3z[kThreads] = dBr[0]; c3z[2 * kThreads] = dBr[1];
        }
        // a rolled two-iteration loop: half the code of an unrolled pair of
        // rows, which keeps the hot path inside the instruction cache
#pragma unroll 1
        for (int q = 0; q < 2; ++q) {
            const int r = rr + q;
            const int gi = x0 + r;
            const int g = gi * P + (z0 + c);
            // the leapfrog's operands first: their latency runs under the derivatives
            const float4 npx = ldg4(nowp[0] + g), npz = ldg4(nowp[1] + g);
            const float4 nsx = ldg4(nowp[2] + g), nsz = ldg4(nowp[3] + g);
            const float4 opx = ldg4(p.past[0] + off + g), opz = ldg4(p.past[1] + off + g);
            const float4 osx = ldg4(p.past[2] + off + g), osz = ldg4(p.past[3] + off + g);
            float4 tx[1], wx[1], dB[1], dE[1];
            if constexpr (kCarry) {
                tx[0] = txr[0]; wx[0] = wxr[0]; dB[0] = dBr[0]; dE[0] = dEr[0];
                txr[0] = txr[1]; wxr[0] = wxr[1]; dBr[0] = dBr[1]; dEr[0] = dEr[1];
            } else if constexpr (kShare4) {
                tx[0] = c4x[q * kThreads]; wx[0] = c4x[(2 + q) * kThreads];
                dB[0] = c4z[q * kThreads]; dE[0] = c4z[(2 + q) * kThreads];
            } else if constexpr (kShare3) {
                tx[0] = c3x[q * kThreads]; wx[0] = q ? c3z[0] : c3x[2 * kThreads]; dB[0] = c3z[(1 + q) * kThreads];
                dx4<N, 1, true>(sQzz + (r + SHX) * TZ + c, TZ, a, dvx, dE);      // duz_zdx = D+x Qzz
            } else {
                dx4<N, 1, true>(sTh + (r + SHX) * SC + scol, SC, a, dvx, tx);    // dthetadx = D+x theta
                dx4<N, 1, false>(sOm + (r + SHX) * SC + scol, SC, a, dvx, wx);   // domegadx = D-x omega
                dx4<N, 1, false>(sQxz + (r + SHX) * TZ + c, TZ, a, dvx, dB);     // dux_zdx = D-x Qxz
                dx4<N, 1, true>(sQzz + (r + SHX) * TZ + c, TZ, a, dvx, dE);      // duz_zdx = D+x Qzz
            }
            const float4 tz = dz4<N, true>(sTh + (r + SHX) * SC + scol, a, dvz);    // dthetadz
            const float4 wz = dz4<N, false>(sOm + (r + SHX) * SC + scol, a, dvz);   // domegadz
            const float4 dA = dz4<N, true>(sQxx + r * SC + scol, a, dvz);           // dux_xdz = D+z Qxx
            const float4 dC = dz4<N, false>(sQzx + r * SC + scol, a, dvz);          // duz_xdz = D-z Qzx
            float4 oC = zero4(), oE = zero4(), oB = zero4(), oA = zero4();
            float4 oTx = zero4(), oTz = zero4(), oWz = zero4(), oWx = zero4();
            if (f.pz) {
                const float4 d = ldg4(gm.az + g);
                oC = cpml4(ldg4(p.o[0] + off + g), d, dC, dt);
                oA = cpml4(ldg4(p.o[3] + off + g), d, dA, dt);
                oTz = cpml4(ldg4(p.o[5] + off + g), d, tz, dt);
                oWz = cpml4(ldg4(p.o[6] + off + g), d, wz, dt);
            }
            if (f.px) {
                const float4 d = ldg4(gm.ax + g);
                oE = cpml4(ldg4(p.o[1] + off + g), d, dE[0], dt);
                oB = cpml4(ldg4(p.o[2] + off + g), d, dB[0], dt);
                oTx = cpml4(ldg4(p.o[4] + off + g), d, tx[0], dt);
                oWx = cpml4(ldg4(p.o[7] + off + g), d, wx[0], dt);
            }
            // leapfrog brackets in the reference's order (PS:291-294); zero
            // memories outside the damping layers change no rounding
            const float4 nwx = make_float4(-wx[0].x, -wx[0].y, -wx[0].z, -wx[0].w);
            float4 spx = add4(sub4(sub4(add4(sub4(tx[0], oTx), dC), dE[0]), oC), oE);
            float4 spz = add4(sub4(sub4(add4(sub4(tz, oTz), dB[0]), dA), oB), oA);
            float4 ssx = add4(sub4(sub4(add4(sub4(wz, oWz), dC), dE[0]), oC), oE);
            float4 ssz = add4(sub4(sub4(add4(add4(nwx, oWx), dB[0]), dA), oB), oA);
            if (p.density) {   // variable density: acceleration = buoyancy x stress divergence
                const float4 bxv = ldg4(gm.bx + g), bzv = ldg4(gm.bz + g);
                spx = mul4(spx, bxv); ssx = mul4(ssx, bxv);
                spz = mul4(spz, bzv); ssz = mul4(ssz, bzv);
            }
            const float2 two = dup2(2.f), dt2 = dup2(p.dt2), m1 = dup2(-1.f);
            auto leap = [&](float4 now, float4 past, float4 sum) {
                return cat4(fma2(dt2, lo2(sum), fma2(two, lo2(now), mul2(lo2(past), m1))),
                            fma2(dt2, hi2(sum), fma2(two, hi2(now), mul2(hi2(past), m1))));
            };
            float4 vpx = leap(npx, opx, spx), vpz = leap(npz, opz, spz);
            float4 vsx = leap(nsx, osx, ssx), vsz = leap(nsz, osz, ssz);
            if (MODE == kFwd && f.src && sv.src_type == 1 && gi == sv.sx && sv.sz >= z0 + c && sv.sz < z0 + c + 4)
                set_comp(vpz, sv.sz - z0 - c, comp(vpz, sv.sz - z0 - c) + p.dt2 * sv.wavelet[p.t]);
            unsigned live = 0xfu;
            if (f.border) {
                live = 0u;
#pragma unroll
                for (int k = 0; k < 4; ++k) live |= u_live<N, MODE>(p, gm, gi, z0 + c + k) ? (1u << k) : 0u;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (!(live & (1u << k))) {
                        set_comp(vpx, k, 0.f); set_comp(vpz, k, 0.f); set_comp(vsx, k, 0.f); set_comp(vsz, k, 0.f);
                        set_comp(oC, k, 0.f); set_comp(oE, k, 0.f); set_comp(oB, k, 0.f); set_comp(oA, k, 0.f);
                        set_comp(oTx, k, 0.f); set_comp(oTz, k, 0.f); set_comp(oWz, k, 0.f); set_comp(oWx, k, 0.f);
                    }
                }
            }
            if (MODE == kFwd) {
                const float4 ux = add4(vpx, vsx), uz = add4(vpz, vsz);   // PS:302-303
                if (sv.rec_x && sv.rz >= z0 + c && sv.rz < z0 + c + 4 && gi < gm.X) {
                    sv.rec_x[gi] = comp(ux, sv.rz - z0 - c);   // post-update value (PS:307-311)
                    sv.rec_z[gi] = comp(uz, sv.rz - z0 - c);
                }
                if (f.ring) {   // kept for the strip pass below (the U box is free now)
                    st4(sUx + r * TZ + c, ux);
                    st4(sUz + r * TZ + c, uz);
                }
            }
            if (MODE == kRec) {
                // zero-lag imaging condition (corr_v, PS:1426-1439) on the interior
                const float4 sx = p.img_past ? opx : npx;
                const float4 sz = p.img_past ? opz : npz;
                const float4 rpx = ldg4(p.rcv[0] + off + g), rpz = ldg4(p.rcv[1] + off + g);
                const float4 rsx = ldg4(p.rcv[2] + off + g), rsz = ldg4(p.rcv[3] + off + g);
                float* acc0 = p.acc[0] + off + g;
                float* acc1 = p.acc[1] + off + g;
                float* acc2 = p.acc[2] + off + g;
                auto corr = [&](float4 acc, float4 a1, float4 b1, float4 a2, float4 b2) {
                    return cat4(add2(lo2(acc), fma2(lo2(a1), lo2(b1), mul2(lo2(a2), lo2(b2)))),
                                add2(hi2(acc), fma2(hi2(a1), hi2(b1), mul2(hi2(a2), hi2(b2)))));
                };
                const float4 o0 = ldg4(acc0), o1 = ldg4(acc1), o2 = ldg4(acc2);
                if (!p.comp_image) {
                    float4 npp = corr(o0, sx, rpx, sz, rpz);
                    float4 nil = corr(o2, sx, sx, sz, sz);
                    float4 nps = corr(o1, sx, rsx, sz, rsz);
                    if (f.border) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            if (!(live & (1u << k))) {
                                set_comp(npp, k, comp(o0, k)); set_comp(nps, k, comp(o1, k)); set_comp(nil, k, comp(o2, k));
                            }
                        }
                    }
                    stg4(acc0, npp); stg4(acc1, nps); stg4(acc2, nil);
                } else {
                    // compensated sums (Kahan, CACM 8(1), 1965): acc + c carries the
                    // sum to about twice float precision; c holds minus the
                    // low-order part lost by the last addition
                    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
                    const float4 tpp = corr(zero, sx, rpx, sz, rpz), tps = corr(zero, sx, rsx, sz, rsz);
                    const float4 til = corr(zero, sx, sx, sz, sz);
                    float* cp[3] = {p.comp[0] + off + g, p.comp[1] + off + g, p.comp[2] + off + g};
                    const float4 term[3] = {tpp, tps, til}, old[3] = {o0, o1, o2};
                    float* accp[3] = {acc0, acc1, acc2};
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const float4 cq = ldg4(cp[q]);
                        float4 na = old[q], nc = cq;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            if (f.border && !(live & (1u << k))) continue;
                            const float y = __fsub_rn(comp(term[q], k), comp(cq, k));
                            const float t = __fadd_rn(comp(old[q], k), y);
                            set_comp(nc, k, __fsub_rn(__fsub_rn(t, comp(old[q], k)), y));
                            set_comp(na, k, t);
                        }
                        stg4(accp[q], na);
                        stg4(cp[q], nc);
                    }
                }
            }
            stg4(p.past[0] + off + g, vpx); stg4(p.past[1] + off + g, vpz);
            stg4(p.past[2] + off + g, vsx); stg4(p.past[3] + off + g, vsz);
            if (f.pz) {
                stg4(p.o[0] + off + g, oC); stg4(p.o[3] + off + g, oA);
                stg4(p.o[5] + off + g, oTz); stg4(p.o[6] + off + g, oWz);
            }
            if (f.px) {
                stg4(p.o[1] + off + g, oE); stg4(p.o[2] + off + g, oB);
                stg4(p.o[4] + off + g, oTx); stg4(p.o[7] + off + g, oWx);
            }
        }
    }
    if (MODE == kFwd && f.ring) {
        // save_wavefiled (PS:1230-1287): the new displacement of the tile's ring cells
        __syncthreads();
        const ShotDesc& d = p.shots[sv.b];
        void* s = strip_save_ptr(p, d);
        float m[2] = {0.f, 0.f};
        for_ring(gm.ring, x0, x0 + TX, z0, z0 + TZ, [&](int i, int j, int ri) {
            const int o = (i - x0) * TZ + (j - z0);
            const float ux = sUx[o], uz = sUz[o];
            strip_put(p, s, kSUx * R + ri, ux);
            strip_put(p, s, kSUz * R + ri, uz);
            m[0] = fmaxf(m[0], fabsf(ux));
            m[1] = fmaxf(m[1], fabsf(uz));
        });
        if (p.strip_prec == kStripF16) {
            amax_commit<2>(d.amax + (size_t)p.t * kStripFields, kSUx, m);
            if (p.t > 0) {
                // slot t-1 is complete (its maxima with it): convert this tile's
                // cells of it from the staging ring to scaled halves
                const float* src = d.stage + (size_t)((p.t - 1) & 1) * d.strip_slot;
                __half* dst = reinterpret_cast<__half*>(static_cast<char*>(d.strips) + (size_t)(p.t - 1) * slot_bytes(p, d));
                const unsigned* am = d.amax + (size_t)(p.t - 1) * kStripFields;
                int k[kStripFields];
#pragma unroll
                for (int q = 0; q < kStripFields; ++q) k[q] = f16_exp(am[q]);
                for_ring(gm.ring, x0, x0 + TX, z0, z0 + TZ, [&](int, int, int ri) {
                    float v[kStripFields];   // all loads before the stores
#pragma unroll
                    for (int q = 0; q < kStripFields; ++q) v[q] = src[q * R + ri];
#pragma unroll
                    for (int q = 0; q < kStripFields; ++q) dst[q * R + ri] = __float2half_rn(scale2(v[q], k[q]));
                });
            }
        }
    }
    return true;
}

template <int N, int MODE>
__global__ void __launch_bounds__(kThreads, 2) k_step(const __grid_constant__ StepArgs p) {
    extern __shared__ __align__(128) float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    using G = TileGeo<N>;
    const int tz = blockIdx.x % p.tiles_z, tx = blockIdx.x / p.tiles_z;
    const int x0 = p.tile_x0 + tx * G::TX, z0 = p.tile_z0 + tz * G::TZ;
    if (MODE != kRec && x0 >= p.X - N) {
        // every row of the tile lies outside the update domain [N, X-N) of
        // the forward and receiver steps: its cells are never written (they
        // were zeroed with the shot's state), so only the forward's record
        // samples of these rows, zeros, are stored (PS:307-311 records every x)
        if (MODE == kFwd && p.record) {
            const ShotDesc& d = p.shots[blockIdx.y];
            if (d.rz >= z0 && d.rz < z0 + G::TZ)
                for (int i = x0 + (int)threadIdx.x; i < min(x0 + G::TX, d.X); i += kThreads) {
                    d.gather_x[(size_t)p.t * d.X + i] = 0.f;
                    d.gather_z[(size_t)p.t * d.X + i] = 0.f;
                }
        }
        return;
    }
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {   // the tile's copies first: they overlap everything up to phase 1
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issue_u_box<N>(p, sm, x0, z0, blockIdx.y, &bar);
    }
    const ShotDesc& d = p.shots[blockIdx.y];
    if ((int)blockIdx.x >= (MODE == kRec ? d.rec_tiles_x : d.tiles_x) * p.tiles_z) {
        // beyond this shot's width (per-shot sub-grids): the copies (of cells
        // outside the shot's grid) land before the shared memory is released
        if (threadIdx.x == 0) mbar_wait(&bar, 0u);
        return;
    }
    const Geo gm = geo_of(d);
    const ShotView sv = shot_view(p, blockIdx.y);
    const TileFlags f = tile_flags<N, MODE>(p, gm, sv, x0, z0);
    prefetch_tile<N, MODE>(p, gm, x0, z0, blockIdx.y, f);
    if (MODE == kRec && f.ring) prefetch_ring<N>(p, gm, d, x0, z0);
    __syncthreads();   // the mbarrier is initialised
    step_tile<N, MODE>(p, gm, sv, sm, x0, z0, f, &bar, 0u);
}

// The same step as a persistent launch with a dynamic work queue: a few
// CTAs per SM claim (tile, shot) items from a device counter until the
// queue is empty.  Items are ordered heaviest first -- the tiles that meet
// the damping layers (CPML memories) and the boundary ring (strips) lead,
// per the host-built table p.order -- so the cheap interior tiles fill the
// end of the launch.  Each CTA claims its next item while it works on the
// current one and prefetches that tile's operands to L2 right after it has
// its index.  The last CTA to finish resets the counters for the next
// launch of the same mode (no memset per launch).  The queue has no waits:
// a CTA only atomically increments the counter and reads its value (the
// tile's own copy wait is bounded, as in k_step).
template <int N, int MODE>
__global__ void __launch_bounds__(kThreads, 2) k_step_q(const __grid_constant__ StepArgs p, int nshots, int ntiles) {
    extern __shared__ __align__(128) float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    __shared__ int s_item[2];
    using G = TileGeo<N>;
    int* counter = p.queue + 2 * MODE;
    int* done = counter + 1;
    const int* order = p.order[MODE == kRec ? 1 : 0];
    const int nitems = ntiles * nshots;
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        s_item[0] = atomicAdd(counter, 1);
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int item = s_item[0], buf = 0;
    unsigned parity = 0;   // phase of the mbarrier that the next tile's copies complete
    while (item < nitems) {
        if (threadIdx.x == 0) s_item[buf ^ 1] = atomicAdd(counter, 1);
        const int b = item % nshots, k = item / nshots;
        const int tx = order[k] >> 16, tz = order[k] & 0xffff;
        const ShotDesc& d = p.shots[b];
        if (tx < (MODE == kRec ? d.rec_tiles_x : d.tiles_x)) {   // within this shot's width
            const int x0 = p.tile_x0 + tx * G::TX, z0 = p.tile_z0 + tz * G::TZ;
            if (threadIdx.x == 0) issue_u_box<N>(p, sm, x0, z0, b, &bar);
            const Geo gm = geo_of(d);
            const ShotView sv = shot_view(p, b);
            const TileFlags f = tile_flags<N, MODE>(p, gm, sv, x0, z0);
            prefetch_tile<N, MODE>(p, gm, x0, z0, b, f);
            if (MODE == kRec && f.ring) prefetch_ring<N>(p, gm, d, x0, z0);
            if (!step_tile<N, MODE>(p, gm, sv, sm, x0, z0, f, &bar, parity)) break;   // uniform: reported
            parity ^= 1u;
        }
        __syncthreads();   // the tile's shared memory is free and the next index is visible
        item = s_item[buf ^ 1];
        buf ^= 1;
    }
    if (threadIdx.x == 0) {
        __threadfence();   // this CTA's claims are complete before it counts itself done
        if (atomicAdd(done, 1) == (int)gridDim.x - 1) {
            *counter = 0;
            *done = 0;
            __threadfence();
        }
    }
}

}  // namespace ouc
