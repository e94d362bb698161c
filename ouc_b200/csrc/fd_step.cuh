// Fused time-step kernel of the elastic P/S-decoupled staggered-grid
// scheme (sm_100a).
//
// One launch advances one wavefield by one time step.  The reference does it
// in two launches that talk through six full-grid HBM arrays (forward_s then
// forward_u, PS:2261-2264; rt_s_res/rt_u_res; reshot_u/reshot_s).  Here each
// CTA owns a TX x TZ tile of cells and, in three phases separated by
// __syncthreads():
//   1. loads the total displacement U = P + S of its tile plus a 2N halo
//      into shared memory (float4 loads along the contiguous z axis);
//   2. computes the S-stage (theta, omega and the four Q fields, with the
//      S-stage CPML memory) for its tile plus an N halo, keeping it on chip
//      -- the halo cells are recomputed by both neighbouring CTAs, so the six
//      intermediate fields never reach HBM;
//   3. computes the U-stage for its own cells: eight staggered derivatives of
//      the S fields, U-stage CPML memory, the P/S leapfrog, and writes the
//      new level over the oldest one (ping-pong of the P/S pairs makes the
//      halo reads of phase 1 race-free).
// Receiver extraction, record injection, boundary-strip save/restore and the
// zero-lag imaging condition ride along in the same launch.
//
// Arithmetic follows the reference operation by operation (coefficient sums
// in k order then divided by the spacing, PS:229; the CPML update form of
// PS:281; the leapfrog bracket order of PS:291-294), and memory terms that
// are identically zero outside the damping layers are skipped, which leaves
// every rounding unchanged.
#pragma once
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

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float comp(const float4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(float4& v, int k, float x) {
    if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
}

// CPML memory update m + (d*e - d*m)*dt, the form of PS:281 and PS:368.
__device__ __forceinline__ float cpml1(float m, float d, float e, float dt) { return m + (d * e - d * m) * dt; }

// Staggered derivative of four consecutive z cells starting at `row`
// (16-byte aligned shared-memory pointer at the first of the four cells).
// PLUS: sum_k a_k (f[j+k] - f[j-k+1]);  MINUS: sum_k a_k (f[j+k-1] - f[j-k]).
template <int N, bool PLUS>
__device__ __forceinline__ float4 dz4(const float* row, const float* a, float h) {
    constexpr int NB = (N + 3) / 4;
    float w[4 * (2 * NB + 1)];
#pragma unroll
    for (int b = 0; b < 2 * NB + 1; ++b) {
        float4 v = ld4(row + 4 * (b - NB));
        w[4 * b + 0] = v.x; w[4 * b + 1] = v.y; w[4 * b + 2] = v.z; w[4 * b + 3] = v.w;
    }
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int c = 4 * NB + q;
        float acc = PLUS ? a[0] * (w[c + 1] - w[c]) : a[0] * (w[c] - w[c - 1]);
#pragma unroll
        for (int k = 1; k < N; ++k)
            acc = PLUS ? acc + a[k] * (w[c + k + 1] - w[c - k]) : acc + a[k] * (w[c + k] - w[c - k - 1]);
        o[q] = acc / h;
    }
    return make_float4(o[0], o[1], o[2], o[3]);
}

// Staggered x derivatives of RR consecutive rows of one float4 column.
// `col` points at row r0 of the column in shared memory, `st` is the row
// stride in floats.  Window rows r0-N .. r0+RR-1+N are read once.
template <int N, int RR, bool PLUS>
__device__ __forceinline__ void dx4(const float* col, int st, const float* a, float h, float4 (&out)[RR]) {
    float4 w[RR + 2 * N];
#pragma unroll
    for (int k = 0; k < RR + 2 * N; ++k) {
        if (PLUS ? k >= 1 : k < RR + 2 * N - 1) w[k] = ld4(col + (k - N) * st);
    }
#pragma unroll
    for (int q = 0; q < RR; ++q) {
        const int c = q + N;
        float4 acc;
        if (PLUS) {
            acc.x = a[0] * (w[c + 1].x - w[c].x); acc.y = a[0] * (w[c + 1].y - w[c].y);
            acc.z = a[0] * (w[c + 1].z - w[c].z); acc.w = a[0] * (w[c + 1].w - w[c].w);
        } else {
            acc.x = a[0] * (w[c].x - w[c - 1].x); acc.y = a[0] * (w[c].y - w[c - 1].y);
            acc.z = a[0] * (w[c].z - w[c - 1].z); acc.w = a[0] * (w[c].w - w[c - 1].w);
        }
#pragma unroll
        for (int k = 1; k < N; ++k) {
            const int hi = PLUS ? c + k + 1 : c + k, lo = PLUS ? c - k : c - k - 1;
            acc.x = acc.x + a[k] * (w[hi].x - w[lo].x);
            acc.y = acc.y + a[k] * (w[hi].y - w[lo].y);
            acc.z = acc.z + a[k] * (w[hi].z - w[lo].z);
            acc.w = acc.w + a[k] * (w[hi].w - w[lo].w);
        }
        out[q] = make_float4(acc.x / h, acc.y / h, acc.z / h, acc.w / h);
    }
}

template <int N, int MODE, bool PX, bool PZ>
__device__ __forceinline__ void step_tile(const StepArgs& p, float* sm, int x0, int z0) {
    using G = TileGeo<N>;
    constexpr int TX = G::TX, TZ = G::TZ, SHX = G::SHX, HS = G::HS, HU = G::HU, UC = G::UC, SC = G::SC;
    const int tid = threadIdx.x;
    const int X = p.X, Z = p.Z, P = p.pitch, L = p.L;
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

    // ---- phase 1: U = P + S over the tile and a 2N halo ---------------------
    for (int idx = tid; idx < G::UR * (UC / 4); idx += kThreads) {
        const int r = idx / (UC / 4), c4 = idx - r * (UC / 4);
        const int gi = x0 - SHX - N + r, gj = z0 - HU + 4 * c4;
        const ptrdiff_t g = (ptrdiff_t)gi * P + gj;
        const float4 px = ld4(p.now[0] + g), pz = ld4(p.now[1] + g);
        const float4 qx = ld4(p.now[2] + g), qz = ld4(p.now[3] + g);
        float4 ux = make_float4(px.x + qx.x, px.y + qx.y, px.z + qx.z, px.w + qx.w);
        float4 uz = make_float4(pz.x + qz.x, pz.y + qz.y, pz.z + qz.z, pz.w + qz.w);
        if (MODE == kRcv) {
            // load_record (PS:1471-1483): the receiver row is overwritten by the
            // record over the interior x range before the S-stage reads it
            if (p.inj_x && gi >= L && gi < X - L && p.rz >= gj && p.rz < gj + 4) {
                set_comp(ux, p.rz - gj, p.inj_x[gi]);
                set_comp(uz, p.rz - gj, p.inj_z[gi]);
            }
        }
        if (MODE == kRec) {
            // reconstruction: the ring comes from the saved strips, cells
            // outside the box are never read by the interior update
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int j = gj + k;
                float vx = comp(ux, k), vz = comp(uz, k);
                if (!p.ring.in_box(gi, j)) {
                    vx = 0.f; vz = 0.f;
                } else {
                    const int ri = p.ring.index(gi, j);
                    if (ri >= 0) {
                        vx = p.strip_u[(size_t)kSUx * p.ring.R + ri];
                        vz = p.strip_u[(size_t)kSUz * p.ring.R + ri];
                    }
                }
                set_comp(ux, k, vx); set_comp(uz, k, vz);
            }
        }
        st4(sUx + r * UC + 4 * c4, ux);
        st4(sUz + r * UC + 4 * c4, uz);
    }
    __syncthreads();

    // ---- phase 2: S-stage on the tile plus an N halo -------------------------
    if (tid < G::itemsA + G::itemsB) {
        int r0, c;
        bool groupA = tid < G::itemsA;
        if (groupA) {
            r0 = -SHX + 4 * (tid / (TZ / 4));
            c = 4 * (tid % (TZ / 4));
        } else {
            const int k = tid - G::itemsA;
            r0 = 4 * (k / (2 * HS / 4));
            const int cc = k % (2 * HS / 4);
            c = cc < HS / 4 ? -HS + 4 * cc : TZ + 4 * (cc - HS / 4);
        }
        // U shared-memory coordinates of (r0, c)
        const float* ux0 = sUx + (r0 + SHX + N) * UC + (c + HU);
        const float* uz0 = sUz + (r0 + SHX + N) * UC + (c + HU);
        float4 exx[4], ezx[4];
        dx4<N, 4, false>(ux0, UC, a, p.dx, exx);   // dvxdx = D-x Ux
        dx4<N, 4, true>(uz0, UC, a, p.dx, ezx);    // dvzdx = D+x Uz
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r0 + q;
            const int gi = x0 + r;
            const int gjb = z0 + c;
            const float4 exz = dz4<N, true>(ux0 + q * UC, a, p.dz);    // dvxdz = D+z Ux
            const float4 ezz = dz4<N, false>(uz0 + q * UC, a, p.dz);   // dvzdz = D-z Uz
            const ptrdiff_t g = (ptrdiff_t)gi * P + gjb;
            const float4 vp2 = ld4(p.vp2 + g), vs2 = ld4(p.vs2 + g);
            const bool own = r >= 0 && r < TX && c >= 0 && c < TZ;
            float4 fo[4], fn[4];
            float4 axv = make_float4(0.f, 0.f, 0.f, 0.f), azv = axv;
            if (PX) { axv = ld4(p.ax + g); fo[0] = ld4(p.f_old[0] + g); fo[3] = ld4(p.f_old[3] + g); }
            if (PZ) { azv = ld4(p.az + g); fo[1] = ld4(p.f_old[1] + g); fo[2] = ld4(p.f_old[2] + g); }
            float4 th, om, qzx, qzz, qxx, qxz;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int gj = gjb + k;
                const float e_xx = comp(exx[q], k), e_zx = comp(ezx[q], k);
                const float e_xz = comp(exz, k), e_zz = comp(ezz, k);
                const float vp2k = comp(vp2, k), vs2k = comp(vs2, k);
                float fxx = 0.f, fzz = 0.f, fxz = 0.f, fzx = 0.f;
                if (PX) {
                    fxx = cpml1(comp(fo[0], k), comp(axv, k), e_xx, p.dt);
                    fzx = cpml1(comp(fo[3], k), comp(axv, k), e_zx, p.dt);
                }
                if (PZ) {
                    fzz = cpml1(comp(fo[1], k), comp(azv, k), e_zz, p.dt);
                    fxz = cpml1(comp(fo[2], k), comp(azv, k), e_xz, p.dt);
                }
                float sth = e_xx + e_zz;
                if (PX) sth = sth - fxx;
                if (PZ) sth = sth - fzz;
                float som = e_xz - e_zx;
                if (PZ) som = som - fxz;
                if (PX) som = som + fzx;
                float v_th = vp2k * sth;
                float v_om = vs2k * som;
                float v_qzx = vs2k * (PX ? e_zx - fzx : e_zx);
                float v_qzz = vs2k * (PZ ? e_zz - fzz : e_zz);
                float v_qxz = vs2k * (PZ ? e_xz - fxz : e_xz);
                float v_qxx = vs2k * (PX ? e_xx - fxx : e_xx);
                bool live;
                if (MODE == kRec) {
                    live = p.ring.in_box(gi, gj);
                    if (live && p.src_recon && gi == p.sx && gj == p.sz) v_th = v_th + p.wavelet[p.src_t];
                    const int ri = live ? p.ring.index(gi, gj) : -1;
                    if (ri >= 0) {
                        const float* s = p.strip_s;
                        const size_t R = p.ring.R;
                        v_th = s[kSTh * R + ri]; v_om = s[kSOm * R + ri];
                        v_qzx = s[kSQzx * R + ri]; v_qzz = s[kSQzz * R + ri];
                        v_qxx = s[kSQxx * R + ri]; v_qxz = s[kSQxz * R + ri];
                    }
                } else {
                    live = gi >= N && gi < X - N && gj >= N && gj < Z - N;
                    if (MODE == kFwd && p.src_type == 0 && gi == p.sx && gj == p.sz) v_th = v_th + p.wavelet[p.src_t];
                }
                if (!live) {
                    v_th = v_om = v_qzx = v_qzz = v_qxz = v_qxx = 0.f;
                    fxx = fzz = fxz = fzx = 0.f;
                }
                set_comp(th, k, v_th); set_comp(om, k, v_om);
                set_comp(qzx, k, v_qzx); set_comp(qzz, k, v_qzz);
                set_comp(qxx, k, v_qxx); set_comp(qxz, k, v_qxz);
                if (PX) { set_comp(fn[0], k, fxx); set_comp(fn[3], k, fzx); }
                if (PZ) { set_comp(fn[1], k, fzz); set_comp(fn[2], k, fxz); }
                if (MODE == kFwd && own && p.strip_save) {
                    const int ri = p.ring.index(gi, gj);
                    if (ri >= 0) {
                        float* s = p.strip_save;
                        const size_t R = p.ring.R;
                        s[kSTh * R + ri] = v_th; s[kSOm * R + ri] = v_om;
                        s[kSQzx * R + ri] = v_qzx; s[kSQzz * R + ri] = v_qzz;
                        s[kSQxx * R + ri] = v_qxx; s[kSQxz * R + ri] = v_qxz;
                    }
                }
            }
            if (own) {
                if (PX) { st4(p.f_new[0] + g, fn[0]); st4(p.f_new[3] + g, fn[3]); }
                if (PZ) { st4(p.f_new[1] + g, fn[1]); st4(p.f_new[2] + g, fn[2]); }
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
    __syncthreads();

    // ---- phase 3: U-stage on the tile's own cells (2 rows x 4 columns) ------
    {
        const int rr = 2 * (tid / (TZ / 4));
        const int c = 4 * (tid % (TZ / 4));
        const int scol = c + HS;
        float4 tx[2], wx[2], dB[2], dE[2];
        dx4<N, 2, true>(sTh + (rr + SHX) * SC + scol, SC, a, p.dx, tx);    // dthetadx = D+x theta
        dx4<N, 2, false>(sOm + (rr + SHX) * SC + scol, SC, a, p.dx, wx);   // domegadx = D-x omega
        dx4<N, 2, false>(sQxz + (rr + SHX) * TZ + c, TZ, a, p.dx, dB);     // dux_zdx = D-x Qxz
        dx4<N, 2, true>(sQzz + (rr + SHX) * TZ + c, TZ, a, p.dx, dE);      // duz_zdx = D+x Qzz
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int r = rr + q;
            const int gi = x0 + r;
            const ptrdiff_t g = (ptrdiff_t)gi * P + (z0 + c);
            const float4 tz = dz4<N, true>(sTh + (r + SHX) * SC + scol, a, p.dz);    // dthetadz
            const float4 wz = dz4<N, false>(sOm + (r + SHX) * SC + scol, a, p.dz);   // domegadz
            const float4 dA = dz4<N, true>(sQxx + r * SC + scol, a, p.dz);           // dux_xdz = D+z Qxx
            const float4 dC = dz4<N, false>(sQzx + r * SC + scol, a, p.dz);          // duz_xdz = D-z Qzx
            float4 axv = make_float4(0.f, 0.f, 0.f, 0.f), azv = axv;
            float4 om_[8];
            if (PX) {
                axv = ld4(p.ax + g);
                om_[1] = ld4(p.o[1] + g); om_[2] = ld4(p.o[2] + g);
                om_[4] = ld4(p.o[4] + g); om_[7] = ld4(p.o[7] + g);
            }
            if (PZ) {
                azv = ld4(p.az + g);
                om_[0] = ld4(p.o[0] + g); om_[3] = ld4(p.o[3] + g);
                om_[5] = ld4(p.o[5] + g); om_[6] = ld4(p.o[6] + g);
            }
            const float4 npx = ld4(p.now[0] + g), npz = ld4(p.now[1] + g);
            const float4 nsx = ld4(p.now[2] + g), nsz = ld4(p.now[3] + g);
            const float4 opx = ld4(p.past[0] + g), opz = ld4(p.past[1] + g);
            const float4 osx = ld4(p.past[2] + g), osz = ld4(p.past[3] + g);
            float4 vpx, vpz, vsx, vsz, onew[8];
            float4 rp[4], ac[3];
            if (MODE == kRec) {
                rp[0] = ld4(p.rcv[0] + g); rp[1] = ld4(p.rcv[1] + g); rp[2] = ld4(p.rcv[2] + g); rp[3] = ld4(p.rcv[3] + g);
                ac[0] = ld4(p.acc[0] + g); ac[1] = ld4(p.acc[1] + g); ac[2] = ld4(p.acc[2] + g);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int gj = z0 + c + k;
                const float dtx = comp(tx[q], k), dtz = comp(tz, k), dwx = comp(wx[q], k), dwz = comp(wz, k);
                const float A = comp(dA, k), B = comp(dB[q], k), Cc = comp(dC, k), E = comp(dE[q], k);
                float oC = 0.f, oE = 0.f, oB = 0.f, oA = 0.f, oTx = 0.f, oTz = 0.f, oWz = 0.f, oWx = 0.f;
                if (PZ) {
                    const float d = comp(azv, k);
                    oC = cpml1(comp(om_[0], k), d, Cc, p.dt);
                    oA = cpml1(comp(om_[3], k), d, A, p.dt);
                    oTz = cpml1(comp(om_[5], k), d, dtz, p.dt);
                    oWz = cpml1(comp(om_[6], k), d, dwz, p.dt);
                }
                if (PX) {
                    const float d = comp(axv, k);
                    oE = cpml1(comp(om_[1], k), d, E, p.dt);
                    oB = cpml1(comp(om_[2], k), d, B, p.dt);
                    oTx = cpml1(comp(om_[4], k), d, dtx, p.dt);
                    oWx = cpml1(comp(om_[7], k), d, dwx, p.dt);
                }
                // leapfrog brackets in the reference's order (PS:291-294)
                float spx = dtx, spz = dtz, ssx = dwz, ssz = -dwx;
                if (PX) spx = spx - oTx;
                if (PZ) spz = spz - oTz;
                if (PZ) ssx = ssx - oWz;
                if (PX) ssz = ssz + oWx;
                spx = spx + Cc - E; ssx = ssx + Cc - E;
                spz = spz + B - A; ssz = ssz + B - A;
                if (PZ) { spx = spx - oC; ssx = ssx - oC; }
                if (PX) { spx = spx + oE; ssx = ssx + oE; }
                if (PX) { spz = spz - oB; ssz = ssz - oB; }
                if (PZ) { spz = spz + oA; ssz = ssz + oA; }
                float v_px = 2 * comp(npx, k) - comp(opx, k) + p.dt2 * spx;
                float v_pz = 2 * comp(npz, k) - comp(opz, k) + p.dt2 * spz;
                float v_sx = 2 * comp(nsx, k) - comp(osx, k) + p.dt2 * ssx;
                float v_sz = 2 * comp(nsz, k) - comp(osz, k) + p.dt2 * ssz;
                bool live;
                if (MODE == kRec) live = gi >= L && gi < X - L && gj >= L && gj < Z - L;
                else live = gi >= N && gi < X - N && gj >= N && gj < Z - N;
                if (MODE == kFwd && p.src_type == 1 && live && gi == p.sx && gj == p.sz)
                    v_pz = v_pz + p.dt2 * p.wavelet[p.src_t];
                if (!live) {
                    v_px = v_pz = v_sx = v_sz = 0.f;
                    oC = oE = oB = oA = oTx = oTz = oWz = oWx = 0.f;
                }
                set_comp(vpx, k, v_px); set_comp(vpz, k, v_pz);
                set_comp(vsx, k, v_sx); set_comp(vsz, k, v_sz);
                if (PZ) { set_comp(onew[0], k, oC); set_comp(onew[3], k, oA); set_comp(onew[5], k, oTz); set_comp(onew[6], k, oWz); }
                if (PX) { set_comp(onew[1], k, oE); set_comp(onew[2], k, oB); set_comp(onew[4], k, oTx); set_comp(onew[7], k, oWx); }
                if (MODE != kRcv) {
                    const float v_ux = v_px + v_sx, v_uz = v_pz + v_sz;   // PS:302-303 / PS:978-979
                    if (MODE == kFwd && p.rec_x && gj == p.rz && gi < X) {
                        p.rec_x[gi] = v_ux;   // record the post-update value (PS:307-311)
                        p.rec_z[gi] = v_uz;
                    }
                    if (MODE == kFwd && p.strip_save) {
                        const int ri = p.ring.index(gi, gj);
                        if (ri >= 0) {
                            p.strip_save[(size_t)kSUx * p.ring.R + ri] = v_ux;
                            p.strip_save[(size_t)kSUz * p.ring.R + ri] = v_uz;
                        }
                    }
                }
                if (MODE == kRec) {
                    // zero-lag imaging condition (corr_v, PS:1426-1439) on the interior
                    const float sx_ = p.img_past ? comp(opx, k) : comp(npx, k);
                    const float sz_ = p.img_past ? comp(opz, k) : comp(npz, k);
                    const float rpx = comp(rp[0], k), rpz = comp(rp[1], k), rsx = comp(rp[2], k), rsz = comp(rp[3], k);
                    if (live) {
                        set_comp(ac[0], k, comp(ac[0], k) + (sx_ * rpx + sz_ * rpz));
                        set_comp(ac[2], k, comp(ac[2], k) + (sx_ * sx_ + sz_ * sz_));
                        set_comp(ac[1], k, comp(ac[1], k) + (sx_ * rsx + sz_ * rsz));
                    }
                }
            }
            if (MODE == kRec) {
                st4(p.acc[0] + g, ac[0]); st4(p.acc[1] + g, ac[1]); st4(p.acc[2] + g, ac[2]);
            }
            st4(p.past[0] + g, vpx); st4(p.past[1] + g, vpz);
            st4(p.past[2] + g, vsx); st4(p.past[3] + g, vsz);
            if (PZ) { st4(p.o[0] + g, onew[0]); st4(p.o[3] + g, onew[3]); st4(p.o[5] + g, onew[5]); st4(p.o[6] + g, onew[6]); }
            if (PX) { st4(p.o[1] + g, onew[1]); st4(p.o[2] + g, onew[2]); st4(p.o[4] + g, onew[4]); st4(p.o[7] + g, onew[7]); }
        }
    }
}

template <int N, int MODE>
__global__ void __launch_bounds__(kThreads, 2) k_step(const StepArgs p) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    using G = TileGeo<N>;
    const int tz = blockIdx.x % p.tiles_z, tx = blockIdx.x / p.tiles_z;
    const int x0 = (p.tile_x0 + tx) * G::TX, z0 = (p.tile_z0 + tz) * G::TZ;
    if (MODE == kRec) {
        step_tile<N, MODE, false, false>(p, sm, x0, z0);
        return;
    }
    // Damping is non-zero for i < L or i > X-L (PS:2072-2080); a tile takes
    // the memory-variable path when its S-stage halo touches such a cell.
    const bool px = (x0 - G::SHX < p.L) || (x0 + G::TX + G::SHX - 1 >= p.X - p.L);
    const bool pz = (z0 - G::HS < p.L) || (z0 + G::TZ + G::HS - 1 >= p.Z - p.L);
    if (px && pz) step_tile<N, MODE, true, true>(p, sm, x0, z0);
    else if (px) step_tile<N, MODE, true, false>(p, sm, x0, z0);
    else if (pz) step_tile<N, MODE, false, true>(p, sm, x0, z0);
    else step_tile<N, MODE, false, false>(p, sm, x0, z0);
}

}  // namespace ouc
