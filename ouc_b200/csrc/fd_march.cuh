// x-marching fused time-step kernel (sm_100a): the step kernel's arithmetic
// (fd_step.cuh helpers, bit-identical roundings) reorganised so that every
// cell's S-stage is computed once along x and the global operands of the
// first two phases arrive by bulk asynchronous copies (TMA) one block ahead.
//
// Work item: one shot (blockIdx.y), one z-strip of TZ = 64 columns and one
// x-segment of rows [xs, xe) (blockIdx.x).  The CTA walks the segment in
// blocks of RB = 16 rows.  For the block whose own rows are [o, o + RB):
//   1. build U = P + S for the RB new rows [o + SHX + N, o + RB + SHX + N)
//      from the raw stage (P and S of the current level, brought in by
//      cp.async.bulk row copies completing on an mbarrier);
//   2. the S-stage (theta, omega, the four Q fields, S-stage CPML) for the RB
//      new S rows [o + SHX, o + RB + SHX) over the strip plus a z-halo of HS
//      columns, with the model rows from the second stage;
//   3. the U-stage for the own rows [o, o + RB): x-derivatives over S rows
//      [o - SHX, o + RB + SHX), z-derivatives over the own row;
//   4. shift: the U rows and S rows the next block needs (2N rows of each,
//      N of Qxx/Qzx) move up by RB rows in shared memory (x-windows stay
//      contiguous, no modular indexing).
// Before the first own block, two prologue iterations load the U rows above
// the segment and compute the S rows above it (the x-halo of the segment is
// the only S-stage work done twice).  Between blocks the producer lanes of
// warp 0 issue the next block's row copies as soon as the stage is free.
//
// Waits on the copies are bounded: after ~20 ms of polling the CTA records
// the failure, issues no further copies, gives the copies in flight one more
// bounded wait before it exits and sets bit 0 of *StepArgs::err; every later
// CTA and launch that sees the bit returns at once, and the host reports
// OUC_ETIMEOUT after the call.
#pragma once
#include <cstdint>

#include "fd_step.cuh"

namespace ouc {

template <int N>
struct MarchGeo {
    static constexpr int TZ = 64;                      // strip width (z)
    static constexpr int RB = 16;                      // rows per block (x)
    static constexpr int NT = kThreads;                // one U-stage float4 per thread
    static constexpr int SHX = N;                      // S rows above/below the own rows
    static constexpr int HS = (N + 3) & ~3;            // S-stage column halo
    static constexpr int HU = (HS + N + 3) & ~3;       // U column halo
    static constexpr int UC = TZ + 2 * HU;
    static constexpr int SC = TZ + 2 * HS;
    static constexpr int UR = RB + 2 * N;              // U rows held: [o + SHX - N, o + SHX + RB + N)
    static constexpr int SR = RB + 2 * SHX;            // theta, omega, Qxz, Qzz rows: [o - SHX, o + RB + SHX)
    static constexpr int QR = RB + SHX;                // Qxx, Qzx rows: [o, o + RB + SHX)
    static constexpr int oUx = 0;
    static constexpr int oUz = oUx + UR * UC;
    static constexpr int oTh = oUz + UR * UC;
    static constexpr int oOm = oTh + SR * SC;
    static constexpr int oQxz = oOm + SR * SC;
    static constexpr int oQzz = oQxz + SR * TZ;
    static constexpr int oQxx = oQzz + SR * TZ;
    static constexpr int oQzx = oQxx + QR * SC;
    static constexpr int oRaw = oQzx + QR * SC;        // stage: Px Pz Sx Sz of the RB new U rows
    static constexpr int oMod = oRaw + 4 * RB * UC;    // stage: vp2 vs2 of the RB new S rows
    static constexpr int oBar = oMod + 2 * RB * SC;    // two mbarriers (8 bytes each)
    static constexpr int floats = oBar + 4;
    static constexpr int bytes = floats * 4;
    static constexpr int SCOLS = SC / 4;
    static constexpr int UCOLS = UC / 4;
    static constexpr int sItems = (RB / 2) * SCOLS;    // S-stage items: 2 rows x one float4
    static_assert(RB * (TZ / 4) == NT, "one U-stage item per thread");
    static_assert(sItems <= NT, "one S-stage item per thread");
    static_assert(UR - RB <= RB && SR - RB <= RB && QR - RB <= RB, "shifts copy disjoint row ranges");
    static_assert((UC * 4) % 16 == 0 && (SC * 4) % 16 == 0, "bulk copies move 16-byte multiples");
};

// ---- untiled bulk copies (the mbarrier helpers are in fd_step.cuh) ----------
// One contiguous global -> shared copy (16-byte aligned, 16-byte multiple),
// completing `bytes` of the mbarrier's transaction count.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}

// Issue the raw-stage copies of iteration k (U rows [base, base + RB), the
// four P/S fields of the current level, columns [z0 - HU, z0 + TZ + HU)) from
// the lanes of warp 0.  Rows above the guard band are not copied: they only
// feed S rows that no U-stage uses.
template <int N>
__device__ __forceinline__ void issue_raw(const StepArgs& p, size_t off, int base, int z0, float* stage,
                                          uint64_t* bar, int lane) {
    using G = MarchGeo<N>;
    const int r0 = base < -kGX ? -kGX - base : 0;
    const unsigned bytes = (unsigned)(4 * (G::RB - r0) * G::UC * 4);
    if (lane == 0) mbar_arrive_tx(bar, bytes);
    __syncwarp();
    for (int q = lane; q < 4 * G::RB; q += 32) {
        const int f = q / G::RB, r = q - f * G::RB;
        if (r < r0) continue;
        bulk_g2s(stage + (f * G::RB + r) * G::UC, p.now[f] + off + (ptrdiff_t)(base + r) * p.pitch + (z0 - G::HU),
                 G::UC * 4, bar);
    }
}

// Model rows [base, base + RB) (vp2, vs2), columns [z0 - HS, z0 + TZ + HS).
template <int N>
__device__ __forceinline__ void issue_model(const StepArgs& p, const Geo& gm, int base, int z0, float* stage,
                                            uint64_t* bar, int lane) {
    using G = MarchGeo<N>;
    const int r0 = base < -kGX ? -kGX - base : 0;
    const unsigned bytes = (unsigned)(2 * (G::RB - r0) * G::SC * 4);
    if (lane == 0) mbar_arrive_tx(bar, bytes);
    __syncwarp();
    for (int q = lane; q < 2 * G::RB; q += 32) {
        const int f = q / G::RB, r = q - f * G::RB;
        if (r < r0) continue;
        const float* src = (f ? gm.vs2 : gm.vp2) + (ptrdiff_t)(base + r) * p.pitch + (z0 - G::HS);
        bulk_g2s(stage + (f * G::RB + r) * G::SC, src, G::SC * 4, bar);
    }
}

template <int N, int MODE>
__global__ void __launch_bounds__(kThreads, 2) k_march(const StepArgs p) {
    using G = MarchGeo<N>;
    constexpr int TZ = G::TZ, RB = G::RB, SHX = G::SHX, HS = G::HS, HU = G::HU, UC = G::UC, SC = G::SC;
    constexpr int UR = G::UR, SR = G::SR, QR = G::QR;
    extern __shared__ __align__(128) float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    float* sUx = sm + G::oUx;
    float* sUz = sm + G::oUz;
    float* sTh = sm + G::oTh;
    float* sOm = sm + G::oOm;
    float* sQxz = sm + G::oQxz;
    float* sQzz = sm + G::oQzz;
    float* sQxx = sm + G::oQxx;
    float* sQzx = sm + G::oQzx;
    float* sRaw = sm + G::oRaw;
    float* sMod = sm + G::oMod;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + G::oBar);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // ---- work item --------------------------------------------------------------
    const ShotDesc& d = p.shots[blockIdx.y];
    const int strip = blockIdx.x % p.tiles_z, seg = blockIdx.x / p.tiles_z;
    const int X = d.X, Z = p.Z, L = p.L;
    const int row0 = MODE == kRec ? (L / RB) * RB : 0;
    const int row_end = MODE == kRec ? X - L : (X + RB - 1) / RB * RB;
    const int xs = row0 + seg * p.seg_rows;
    if (xs >= row_end) return;   // beyond this shot's rows
    if (p.err && (*(volatile int*)p.err & 1)) return;   // an earlier copy wait gave up: do nothing more
    const int xe = min(xs + p.seg_rows, row_end);
    const int z0 = p.tile_z0 + strip * TZ;
    const int nblk = (xe - xs + RB - 1) / RB;
    const Geo gm = geo_of(d);
    const ShotView sv = shot_view(p, blockIdx.y);
    const size_t off = sv.off;
    const int P = p.pitch;
    const size_t R = gm.ring.R;
    float a[N];
#pragma unroll
    for (int k = 0; k < N; ++k) a[k] = p.a[k];
    const Div dvx = make_div(p.dx, p.rdx), dvz = make_div(p.dz, p.rdz);

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    __syncthreads();
    // prologue copies: raw rows of iteration -2, model rows of iteration -1
    if (warp == 0) {
        issue_raw<N>(p, off, xs - 2 * RB + SHX + N, z0, sRaw, &bars[0], lane);
        issue_model<N>(p, gm, xs - RB + SHX, z0, sMod, &bars[1], lane);
    }
    bool timed_out = false;
    int nraw = 1, nmod = 1;   // stage phases issued so far (the prologue issued one of each)

    // per-strip flags (uniform over the item)
    const bool pz = z0 - HS < L || z0 + TZ + HS - 1 >= Z - L;        // S region meets the z damping
    const bool pz_own = z0 < L || z0 + TZ - 1 >= Z - L;               // own columns meet it
    const bool rec_here = MODE == kFwd && sv.rec_x && sv.rz >= z0 && sv.rz < z0 + TZ;

#pragma unroll 1
    for (int k = -2; k < nblk; ++k) {
        const int o = xs + k * RB;
        const int ubase = o + SHX + N;   // first new U row
        const int sbase = o + SHX;       // first new S row
        // ---- 1. U = P + S for the new U rows ----------------------------------------
        if (!timed_out && !mbar_wait(&bars[0], (unsigned)(k + 2) & 1u)) timed_out = true;
        for (int idx = tid; idx < RB * G::UCOLS; idx += kThreads) {
            const int r = idx / G::UCOLS, c4 = idx - r * G::UCOLS;
            const float* s = sRaw + r * UC + 4 * c4;
            st4(sUx + (UR - RB + r) * UC + 4 * c4, add4(ld4(s), ld4(s + 2 * RB * UC)));            // Ux = Px + Sx
            st4(sUz + (UR - RB + r) * UC + 4 * c4, add4(ld4(s + RB * UC), ld4(s + 3 * RB * UC)));  // Uz = Pz + Sz
        }
        if (MODE == kRcv && sv.rz >= z0 - HU && sv.rz < z0 + TZ + HU && ubase < X - L && ubase + RB > L) {
            __syncthreads();
            // load_record (PS:1471-1483): the receiver row is overwritten by
            // the record over the interior x range before the S-stage reads it
            const int col = sv.rz - (z0 - HU);
            if (tid < RB) {
                const int gi = ubase + tid;
                if (gi >= L && gi < X - L) {
                    sUx[(UR - RB + tid) * UC + col] = sv.inj_x[gi];
                    sUz[(UR - RB + tid) * UC + col] = sv.inj_z[gi];
                }
            }
        }
        if (MODE == kRec && sv.strips && rect_meets_ring(gm.ring, ubase, ubase + RB, z0 - HU, z0 + TZ + HU)) {
            __syncthreads();
            // reconstruction: the ring comes from the saved strips (read_wavefiled1, PS:1344-1376)
            const void* su = strip_slot_ptr(p, d, p.slot_u);
            const unsigned* am = d.amax ? d.amax + (size_t)p.slot_u * kStripFields : nullptr;
            for_ring(gm.ring, ubase, ubase + RB, z0 - HU, z0 + TZ + HU, [&](int i, int j, int ri) {
                const int oo = (i - ubase + UR - RB) * UC + (j - (z0 - HU));
                sUx[oo] = strip_get(p, su, am, kSUx, kSUx * R + ri);
                sUz[oo] = strip_get(p, su, am, kSUz, kSUz * R + ri);
            });
        }
        timed_out = __syncthreads_or(timed_out);   // uniform over the CTA from here on
        if (k + 1 < nblk && !timed_out) {
            ++nraw;
            if (warp == 0) {
                fence_proxy_async();
                issue_raw<N>(p, off, ubase + RB, z0, sRaw, &bars[0], lane);
            }
        }

        // ---- 2. S-stage on the new S rows ---------------------------------------------
        if (k >= -1) {
            if (!timed_out && !mbar_wait(&bars[1], (unsigned)(k + 1) & 1u)) timed_out = true;
            const bool px = sbase < L || sbase + RB - 1 >= X - L;
            const bool border = MODE != kRec && !(sbase >= N && sbase + RB <= X - N && z0 - HS >= N && z0 + TZ + HS <= Z - N);
            if (tid < G::sItems) {
                const int rp = tid / G::SCOLS;
                const int c = 4 * (tid - rp * G::SCOLS) - HS;   // first column, relative to z0
                const int bs0 = SR - RB + 2 * rp;               // S-buffer row of the first of the two rows
                const bool ownc = c >= 0 && c < TZ;
                // U-buffer row of S row bs: (o - SHX + bs) - (o + SHX - N)
                const float* ux0 = sUx + (bs0 - 2 * SHX + N) * UC + (c + HU);
                const float* uz0 = sUz + (bs0 - 2 * SHX + N) * UC + (c + HU);
                float4 exx[2], ezx[2];
                dx4<N, 2, false>(ux0, UC, a, dvx, exx);   // dvxdx = D-x Ux
                dx4<N, 2, true>(uz0, UC, a, dvx, ezx);    // dvzdx = D+x Uz
#pragma unroll
                for (int qq = 0; qq < 2; ++qq) {
                    const int bs = bs0 + qq;
                    const int gi = o - SHX + bs;
                    const int gjb = z0 + c;
                    const float4 exz = dz4<N, true>(ux0 + qq * UC, a, dvz);    // dvxdz = D+z Ux
                    const float4 ezz = dz4<N, false>(uz0 + qq * UC, a, dvz);   // dvzdz = D-z Uz
                    const int g = gi * P + gjb;
                    const float4 vp2 = ld4(sMod + (2 * rp + qq) * SC + (c + HS));
                    const float4 vs2 = ld4(sMod + (RB + 2 * rp + qq) * SC + (c + HS));
                    const bool own = ownc && gi >= xs && gi < xe;
                    float4 fxx = zero4(), fzz = zero4(), fxz = zero4(), fzx = zero4();
                    if (MODE != kRec && px) {
                        const float4 axv = ld4(gm.ax + g);
                        fxx = cpml4(ld4(p.f_old[0] + off + g), axv, exx[qq], p.dt);
                        fzx = cpml4(ld4(p.f_old[3] + off + g), axv, ezx[qq], p.dt);
                    }
                    if (MODE != kRec && pz) {
                        const float4 azv = ld4(gm.az + g);
                        fzz = cpml4(ld4(p.f_old[1] + off + g), azv, ezz, p.dt);
                        fxz = cpml4(ld4(p.f_old[2] + off + g), azv, exz, p.dt);
                    }
                    // theta = Vp^2 (exx + ezz - Fxx - Fzz), omega = Vs^2 (exz - ezx - Fxz + Fzx)
                    // (PS:373-378); zero memories outside the layers change no rounding
                    float4 th = mul4(vp2, sub4(sub4(add4(exx[qq], ezz), fxx), fzz));
                    float4 om = mul4(vs2, add4(sub4(sub4(exz, ezx[qq]), fxz), fzx));
                    float4 qzx = mul4(vs2, sub4(ezx[qq], fzx));
                    float4 qzz = mul4(vs2, sub4(ezz, fzz));
                    float4 qxz = mul4(vs2, sub4(exz, fxz));
                    float4 qxx = mul4(vs2, sub4(exx[qq], fxx));
                    if (border) {
                        // cells outside [N, X-N) x [N, Z-N) are never updated by the
                        // reference and stay zero
                        const bool row_live = gi >= N && gi < X - N;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int gj = gjb + q;
                            if (!(row_live && gj >= N && gj < Z - N)) {
                                set_comp(th, q, 0.f); set_comp(om, q, 0.f); set_comp(qzx, q, 0.f);
                                set_comp(qzz, q, 0.f); set_comp(qxx, q, 0.f); set_comp(qxz, q, 0.f);
                                set_comp(fxx, q, 0.f); set_comp(fzz, q, 0.f); set_comp(fxz, q, 0.f);
                                set_comp(fzx, q, 0.f);
                            }
                        }
                    }
                    if (MODE != kRec && own) {
                        if (px) { st4(p.f_new[0] + off + g, fxx); st4(p.f_new[3] + off + g, fzx); }
                        if (pz) { st4(p.f_new[1] + off + g, fzz); st4(p.f_new[2] + off + g, fxz); }
                    }
                    st4(sTh + bs * SC + (c + HS), th);
                    st4(sOm + bs * SC + (c + HS), om);
                    if (ownc) {
                        st4(sQxz + bs * TZ + c, qxz);
                        st4(sQzz + bs * TZ + c, qzz);
                    }
                    const int bq = bs - SHX;   // Qxx/Qzx buffer row (row o + bq)
                    st4(sQxx + bq * SC + (c + HS), qxx);
                    st4(sQzx + bq * SC + (c + HS), qzx);
                }
            }
            // source term on theta after the Q fields (PS:380); in the
            // reconstruction only where the level's theta is recomputed
            const bool src_th = MODE == kFwd ? sv.src_type == 0 : (MODE == kRec && p.src_recon);
            if (src_th && sv.sx >= sbase && sv.sx < sbase + RB && sv.sz >= z0 - HS && sv.sz < z0 + TZ + HS) {
                __syncthreads();
                if (tid == 0) {
                    float* t = sTh + (sv.sx - (o - SHX)) * SC + (sv.sz - z0 + HS);
                    *t = *t + sv.wavelet[MODE == kRec ? p.t + 1 : p.t];
                }
            }
            if (MODE == kRec && sv.strips && rect_meets_ring(gm.ring, sbase, sbase + RB, z0 - HS, z0 + TZ + HS)) {
                __syncthreads();
                // read_wavefiled2 (PS:1377-1424): theta, omega and the Q fields of the ring
                const void* ss = strip_slot_ptr(p, d, p.slot_s);
                const unsigned* am = d.amax ? d.amax + (size_t)p.slot_s * kStripFields : nullptr;
                for_ring(gm.ring, sbase, sbase + RB, z0 - HS, z0 + TZ + HS, [&](int i, int j, int ri) {
                    const int bs = i - (o - SHX), c = j - z0;
                    const int so = bs * SC + (c + HS);
                    sTh[so] = strip_get(p, ss, am, kSTh, kSTh * R + ri);
                    sOm[so] = strip_get(p, ss, am, kSOm, kSOm * R + ri);
                    if (c >= 0 && c < TZ) {
                        sQxz[bs * TZ + c] = strip_get(p, ss, am, kSQxz, kSQxz * R + ri);
                        sQzz[bs * TZ + c] = strip_get(p, ss, am, kSQzz, kSQzz * R + ri);
                    }
                    sQxx[(bs - SHX) * SC + (c + HS)] = strip_get(p, ss, am, kSQxx, kSQxx * R + ri);
                    sQzx[(bs - SHX) * SC + (c + HS)] = strip_get(p, ss, am, kSQzx, kSQzx * R + ri);
                });
            }
            const int sa = max(sbase, xs), sb = min(sbase + RB, xe);
            if (MODE == kFwd && p.save && sv.strips && sa < sb && rect_meets_ring(gm.ring, sa, sb, z0, z0 + TZ)) {
                __syncthreads();
                // save_wavefiled (PS:1230-1287): the S fields of the own ring cells
                void* s = strip_save_ptr(p, d);
                float m[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                for_ring(gm.ring, sa, sb, z0, z0 + TZ, [&](int i, int j, int ri) {
                    const int bs = i - (o - SHX), c = j - z0;
                    const int so = bs * SC + (c + HS);
                    const float v[6] = {sTh[so], sOm[so], sQzx[(bs - SHX) * SC + (c + HS)], sQzz[bs * TZ + c],
                                        sQxx[(bs - SHX) * SC + (c + HS)], sQxz[bs * TZ + c]};
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        strip_put(p, s, (kSTh + q) * R + ri, v[q]);
                        m[q] = fmaxf(m[q], fabsf(v[q]));
                    }
                });
                if (p.strip_prec == kStripF16) amax_commit<6>(d.amax + (size_t)p.t * kStripFields, kSTh, m);
            }
        }
        timed_out = __syncthreads_or(timed_out);
        if (k >= -1 && k + 1 < nblk && !timed_out) {
            ++nmod;
            if (warp == 0) {
                fence_proxy_async();
                issue_model<N>(p, gm, sbase + RB, z0, sMod, &bars[1], lane);
            }
        }
        // ---- shift of the U rows: [RB, UR) -> [0, UR - RB) (disjoint ranges; the
        // S-stage has read them, the next U build writes after the closing barrier)
        {
            constexpr int kCarry = (UR - RB) * G::UCOLS;   // float4s per field
            for (int idx = tid; idx < 2 * kCarry; idx += kThreads) {
                const int f = idx / kCarry, e = idx - f * kCarry;
                float* u = f ? sUz : sUx;
                st4(u + 4 * e, ld4(u + RB * UC + 4 * e));
            }
        }

        // ---- 3. U-stage on the own rows [o, o + RB) ------------------------------------
        if (k >= 0) {
            const int r = tid / (TZ / 4);
            const int c = 4 * (tid - r * (TZ / 4));
            const int gi = o + r;
            const bool mine = gi < xe;
            const int bs = r + SHX;   // S-buffer row of the own row
            const int g = gi * P + (z0 + c);
            const float dt = p.dt;
            const bool px_own = o < L || o + RB - 1 >= X - L;
            const bool border = MODE == kRec ? !(o >= L && o + RB <= X - L && z0 >= L && z0 + TZ <= Z - L)
                                             : !(o >= N && o + RB <= X - N && z0 >= N && z0 + TZ <= Z - N);
            // the next block's operands to L2 while this one computes
            if (k + 1 < nblk) {
                const int gn = (gi + RB) * P + (z0 + c);
                if (c % 32 == 0) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(p.past[f] + off + gn));
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(p.now[f] + off + gn));
                        if (MODE == kRec) asm volatile("prefetch.global.L2 [%0];" ::"l"(p.rcv[f] + off + gn));
                    }
                }
            }
            if (mine) {
                const float4 npx = ld4(p.now[0] + off + g), npz = ld4(p.now[1] + off + g);
                const float4 nsx = ld4(p.now[2] + off + g), nsz = ld4(p.now[3] + off + g);
                const float4 opx = ld4(p.past[0] + off + g), opz = ld4(p.past[1] + off + g);
                const float4 osx = ld4(p.past[2] + off + g), osz = ld4(p.past[3] + off + g);
                float4 tx[1], wx[1], dB[1], dE[1];
                dx4<N, 1, true>(sTh + bs * SC + (c + HS), SC, a, dvx, tx);    // dthetadx = D+x theta
                dx4<N, 1, false>(sOm + bs * SC + (c + HS), SC, a, dvx, wx);   // domegadx = D-x omega
                dx4<N, 1, false>(sQxz + bs * TZ + c, TZ, a, dvx, dB);         // dux_zdx = D-x Qxz
                dx4<N, 1, true>(sQzz + bs * TZ + c, TZ, a, dvx, dE);          // duz_zdx = D+x Qzz
                const float4 tz = dz4<N, true>(sTh + bs * SC + (c + HS), a, dvz);    // dthetadz
                const float4 wz = dz4<N, false>(sOm + bs * SC + (c + HS), a, dvz);   // domegadz
                const float4 dA = dz4<N, true>(sQxx + r * SC + (c + HS), a, dvz);    // dux_xdz = D+z Qxx
                const float4 dC = dz4<N, false>(sQzx + r * SC + (c + HS), a, dvz);   // duz_xdz = D-z Qzx
                float4 oC = zero4(), oE = zero4(), oB = zero4(), oA = zero4();
                float4 oTx = zero4(), oTz = zero4(), oWz = zero4(), oWx = zero4();
                if (MODE != kRec && pz_own) {
                    const float4 dd = ld4(gm.az + g);
                    oC = cpml4(ld4(p.o[0] + off + g), dd, dC, dt);
                    oA = cpml4(ld4(p.o[3] + off + g), dd, dA, dt);
                    oTz = cpml4(ld4(p.o[5] + off + g), dd, tz, dt);
                    oWz = cpml4(ld4(p.o[6] + off + g), dd, wz, dt);
                }
                if (MODE != kRec && px_own) {
                    const float4 dd = ld4(gm.ax + g);
                    oE = cpml4(ld4(p.o[1] + off + g), dd, dE[0], dt);
                    oB = cpml4(ld4(p.o[2] + off + g), dd, dB[0], dt);
                    oTx = cpml4(ld4(p.o[4] + off + g), dd, tx[0], dt);
                    oWx = cpml4(ld4(p.o[7] + off + g), dd, wx[0], dt);
                }
                // leapfrog brackets in the reference's order (PS:291-294)
                const float4 nwx = make_float4(-wx[0].x, -wx[0].y, -wx[0].z, -wx[0].w);
                float4 spx = add4(sub4(sub4(add4(sub4(tx[0], oTx), dC), dE[0]), oC), oE);
                float4 spz = add4(sub4(sub4(add4(sub4(tz, oTz), dB[0]), dA), oB), oA);
                float4 ssx = add4(sub4(sub4(add4(sub4(wz, oWz), dC), dE[0]), oC), oE);
                float4 ssz = add4(sub4(sub4(add4(add4(nwx, oWx), dB[0]), dA), oB), oA);
                if (p.density) {   // variable density: acceleration = buoyancy x stress divergence
                    const float4 bxv = ld4(gm.bx + g), bzv = ld4(gm.bz + g);
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
                if (MODE == kFwd && sv.src_type == 1 && gi == sv.sx && sv.sz >= z0 + c && sv.sz < z0 + c + 4)
                    set_comp(vpz, sv.sz - z0 - c, comp(vpz, sv.sz - z0 - c) + p.dt2 * sv.wavelet[p.t]);
                unsigned live = 0xfu;
                if (border) {
                    live = 0u;
#pragma unroll
                    for (int q = 0; q < 4; ++q) live |= u_live<N, MODE>(p, gm, gi, z0 + c + q) ? (1u << q) : 0u;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (!(live & (1u << q))) {
                            set_comp(vpx, q, 0.f); set_comp(vpz, q, 0.f); set_comp(vsx, q, 0.f); set_comp(vsz, q, 0.f);
                            set_comp(oC, q, 0.f); set_comp(oE, q, 0.f); set_comp(oB, q, 0.f); set_comp(oA, q, 0.f);
                            set_comp(oTx, q, 0.f); set_comp(oTz, q, 0.f); set_comp(oWz, q, 0.f); set_comp(oWx, q, 0.f);
                        }
                    }
                }
                if (MODE == kFwd) {
                    const float4 ux = add4(vpx, vsx), uz = add4(vpz, vsz);   // PS:302-303
                    if (rec_here && sv.rz >= z0 + c && sv.rz < z0 + c + 4 && gi < X) {
                        sv.rec_x[gi] = comp(ux, sv.rz - z0 - c);   // post-update value (PS:307-311)
                        sv.rec_z[gi] = comp(uz, sv.rz - z0 - c);
                    }
                    if (p.save && sv.strips && (gm.ring.in_box(gi, z0 + c) || gm.ring.in_box(gi, z0 + c + 3))) {
                        // save_wavefiled (PS:1230-1287): the new displacement of the own ring cells
                        void* s = strip_save_ptr(p, d);
                        float m[2] = {0.f, 0.f};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int ri = gm.ring.index(gi, z0 + c + q);
                            if (ri >= 0) {
                                strip_put(p, s, kSUx * R + ri, comp(ux, q));
                                strip_put(p, s, kSUz * R + ri, comp(uz, q));
                                m[0] = fmaxf(m[0], fabsf(comp(ux, q)));
                                m[1] = fmaxf(m[1], fabsf(comp(uz, q)));
                            }
                        }
                        if (p.strip_prec == kStripF16) {
                            // warp-uniform branch is not guaranteed here: fold per lane
                            unsigned* am = d.amax + (size_t)p.t * kStripFields;
                            if (m[0] > 0.f) atomicMax(am + kSUx, __float_as_uint(m[0]));
                            if (m[1] > 0.f) atomicMax(am + kSUz, __float_as_uint(m[1]));
                        }
                    }
                }
                if (MODE == kRec) {
                    // zero-lag imaging condition (corr_v, PS:1426-1439) on the interior
                    const float4 sx = p.img_past ? opx : npx;
                    const float4 sz = p.img_past ? opz : npz;
                    const float4 rpx = ld4(p.rcv[0] + off + g), rpz = ld4(p.rcv[1] + off + g);
                    const float4 rsx = ld4(p.rcv[2] + off + g), rsz = ld4(p.rcv[3] + off + g);
                    float* acc0 = p.acc[0] + off + g;
                    float* acc1 = p.acc[1] + off + g;
                    float* acc2 = p.acc[2] + off + g;
                    auto corr = [&](float4 acc, float4 a1, float4 b1, float4 a2, float4 b2) {
                        return cat4(add2(lo2(acc), fma2(lo2(a1), lo2(b1), mul2(lo2(a2), lo2(b2)))),
                                    add2(hi2(acc), fma2(hi2(a1), hi2(b1), mul2(hi2(a2), hi2(b2)))));
                    };
                    const float4 o0 = ld4(acc0), o1 = ld4(acc1), o2 = ld4(acc2);
                    if (!p.comp_image) {
                        float4 npp = corr(o0, sx, rpx, sz, rpz);
                        float4 nil = corr(o2, sx, sx, sz, sz);
                        float4 nps = corr(o1, sx, rsx, sz, rsz);
                        if (border) {
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                if (!(live & (1u << q))) {
                                    set_comp(npp, q, comp(o0, q)); set_comp(nps, q, comp(o1, q));
                                    set_comp(nil, q, comp(o2, q));
                                }
                            }
                        }
                        st4(acc0, npp); st4(acc1, nps); st4(acc2, nil);
                    } else {
                        // compensated sums (Kahan, CACM 8(1), 1965)
                        const float4 zero = zero4();
                        const float4 tpp = corr(zero, sx, rpx, sz, rpz), tps = corr(zero, sx, rsx, sz, rsz);
                        const float4 til = corr(zero, sx, sx, sz, sz);
                        float* cp[3] = {p.comp[0] + off + g, p.comp[1] + off + g, p.comp[2] + off + g};
                        const float4 term[3] = {tpp, tps, til}, old[3] = {o0, o1, o2};
                        float* accp[3] = {acc0, acc1, acc2};
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            const float4 cq = ld4(cp[q]);
                            float4 na = old[q], nc = cq;
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                if (border && !(live & (1u << e))) continue;
                                const float y = __fsub_rn(comp(term[q], e), comp(cq, e));
                                const float t = __fadd_rn(comp(old[q], e), y);
                                set_comp(nc, e, __fsub_rn(__fsub_rn(t, comp(old[q], e)), y));
                                set_comp(na, e, t);
                            }
                            st4(accp[q], na);
                            st4(cp[q], nc);
                        }
                    }
                }
                st4(p.past[0] + off + g, vpx); st4(p.past[1] + off + g, vpz);
                st4(p.past[2] + off + g, vsx); st4(p.past[3] + off + g, vsz);
                if (MODE != kRec && pz_own) {
                    st4(p.o[0] + off + g, oC); st4(p.o[3] + off + g, oA);
                    st4(p.o[5] + off + g, oTz); st4(p.o[6] + off + g, oWz);
                }
                if (MODE != kRec && px_own) {
                    st4(p.o[1] + off + g, oE); st4(p.o[2] + off + g, oB);
                    st4(p.o[4] + off + g, oTx); st4(p.o[7] + off + g, oWx);
                }
            }
            if (MODE == kFwd && p.save && sv.strips && p.strip_prec == kStripF16 && p.t > 0) {
                // slot t-1 is complete (its maxima with it): convert this
                // block's own ring cells of it from the staging ring to
                // scaled halves
                const int ra = max(o, xs), rb = min(o + RB, xe);
                if (ra < rb && rect_meets_ring(gm.ring, ra, rb, z0, z0 + TZ)) {
                    const float* src = d.stage + (size_t)((p.t - 1) & 1) * d.strip_slot;
                    __half* dst = reinterpret_cast<__half*>(static_cast<char*>(d.strips) +
                                                            (size_t)(p.t - 1) * slot_bytes(p, d));
                    const unsigned* am = d.amax + (size_t)(p.t - 1) * kStripFields;
                    int ke[kStripFields];
#pragma unroll
                    for (int q = 0; q < kStripFields; ++q) ke[q] = f16_exp(am[q]);
                    for_ring(gm.ring, ra, rb, z0, z0 + TZ, [&](int, int, int ri) {
#pragma unroll
                        for (int q = 0; q < kStripFields; ++q)
                            dst[q * R + ri] = __float2half_rn(scale2(src[q * R + ri], ke[q]));
                    });
                }
            }
        }
        __syncthreads();
        // ---- shift of the S rows: [RB, SR) -> [0, SR - RB), Qxx/Qzx [RB, QR) -> [0, QR - RB)
        {
            constexpr int n1 = (SR - RB) * (SC / 4), n2 = (SR - RB) * (TZ / 4), n3 = (QR - RB) * (SC / 4);
            for (int idx = tid; idx < 2 * n1 + 2 * n2 + 2 * n3; idx += kThreads) {
                float* base;
                int e, w;
                if (idx < 2 * n1) { base = idx < n1 ? sTh : sOm; e = idx < n1 ? idx : idx - n1; w = SC; }
                else if (idx < 2 * n1 + 2 * n2) {
                    const int q = idx - 2 * n1;
                    base = q < n2 ? sQxz : sQzz; e = q < n2 ? q : q - n2; w = TZ;
                } else {
                    const int q = idx - 2 * n1 - 2 * n2;
                    base = q < n3 ? sQxx : sQzx; e = q < n3 ? q : q - n3; w = SC;
                }
                st4(base + 4 * e, ld4(base + RB * w + 4 * e));
            }
        }
    }
    if (timed_out) {
        // no new copies were issued after the failed wait; give the ones in
        // flight a last bounded chance to land before the CTA's shared memory
        // is released, then report
        if (tid == 0) {
            mbar_wait(&bars[0], (unsigned)(nraw - 1) & 1u);
            mbar_wait(&bars[1], (unsigned)(nmod - 1) & 1u);
            if (p.err) atomicOr(p.err, 1);
        }
        __syncthreads();
    }
}

}  // namespace ouc
