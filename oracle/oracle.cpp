// TEST INFRASTRUCTURE -- not part of the product.
//
// CPU oracle for the 2-D elastic P/S-decoupled staggered-grid modeling and
// reverse-time-migration path of gm340/ouc (P-S-seperating.cu, "PS" below).
// It restates, in plain C++ with OpenMP, the kernels that the reference's
// main() actually launches (PS:2258-2376), with the same arithmetic order, so
// that the float instantiation compiled with -ffp-contract=off is bit-exact
// against the reference kernels themselves executed on the CPU
// (oracle/refemu), and the double instantiation is the FP64 oracle every
// result states its error against.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
// this library, and only as a checker or a timed CPU baseline.
//
// Parity is pinned: tests/test_oracle.py compares this file's float
// instantiation bit-for-bit with the reference's own kernels compiled for the
// CPU from the reference sources (oracle/refemu, oracle/Makefile).
//
// Naming: U = total displacement (the reference calls it Vx/Vz), P/S = the
// separated P and S displacement components (Vpx, Vpz, Vsx, Vsz), "now" and
// "past" = the two leapfrog levels, th/om = theta/omega, q.. = the four
// shear-stress-like fields (duzdx=qzx, duzdz=qzz, duxdx=qxx, duxdz=qxz),
// f.. = CPML memory of the S-stage (F_xx ...), o.. = CPML memory of the
// U-stage (O_thetax ...).
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

extern "C" {
// Plain configuration block shared with the Python ctypes wrapper.
typedef struct orc_cfg {
    int X, Z;          // padded grid: X rows (x), Z columns (z, contiguous)
    int L;             // absorbing width; the interior is [L, X-L) x [L, Z-L)
    int N;             // stencil half-width (6 in the reference, PS:16)
    int nt;            // number of time steps (NT, PS:17)
    int sx, sz;        // source cell, padded coordinates (PS:2113)
    int rz;            // receiver row, padded z index (Z_receive, PS:2114)
    int t0;            // wavelet delay in samples, used by the mute (PS:1955)
    int strip_level;   // 0: reference (Vx/Vz strips one level late, PS:2337); 1: exact
    int image_align;   // 0: reference (PS:964 + PS:2361); 1: exact level alignment
    int do_mute;       // 1: apply the direct-wave mute (PS:2293) before back-propagation
    int src_in_recon;  // 1 (exact mode): add the source term inside the reconstruction
    float dx, dz, dt, dh;
    float coeff[8];    // a_1..a_N (PS:221 for N=6)
    int src_type;      // 0: theta source (PS:331-338, 380); 1: vertical force on Uz (no reference counterpart)
} orc_cfg;
}

namespace {

template <class T>
struct Field {
    int X = 0, Z = 0;
    std::vector<T> v;
    void init(int x, int z) { X = x; Z = z; v.assign((size_t)x * z, T(0)); }
    T* p() { return v.data(); }
    const T* p() const { return v.data(); }
    T& operator()(int i, int j) { return v[(size_t)i * Z + j]; }
    T operator()(int i, int j) const { return v[(size_t)i * Z + j]; }
    void zero() { std::fill(v.begin(), v.end(), T(0)); }
};

// Staggered first derivatives, PS:224-279 / PS:340-366.  The coefficient sum
// is accumulated in k order and divided by the spacing afterwards (PS:229).
// dplus:  sum_k a_k (f[c+k] - f[c-k+1]) / h   ("forward" staggering)
// dminus: sum_k a_k (f[c+k-1] - f[c-k]) / h   ("backward" staggering)
template <class T>
inline T dplus(const T* f, ptrdiff_t s, const T* a, int N, T h) {
    T acc = a[0] * (f[s] - f[0]);
    for (int k = 1; k < N; ++k) acc = acc + a[k] * (f[(k + 1) * s] - f[-k * s]);
    return acc / h;
}
template <class T>
inline T dminus(const T* f, ptrdiff_t s, const T* a, int N, T h) {
    T acc = a[0] * (f[0] - f[-s]);
    for (int k = 1; k < N; ++k) acc = acc + a[k] * (f[k * s] - f[-(k + 1) * s]);
    return acc / h;
}
// CPML memory update, PS:281-289 and PS:368-371:  m + (d*e - d*m)*dt
template <class T>
inline T cpml(T m, T d, T e, T dt) { return m + (d * e - d * m) * dt; }

template <class T>
struct Wave {
    int X, Z;
    Field<T> ux, uz;                       // total displacement (Vx, Vz)
    Field<T> pnx, pnz, snx, snz;           // P/S components, level "now"
    Field<T> ppx, ppz, spx, spz;           // P/S components, level "past"
    Field<T> th, om, qzx, qzz, qxx, qxz;   // S-stage outputs
    Field<T> fxx, fzz, fxz, fzx;           // S-stage CPML memory
    Field<T> oC, oE, oB, oA, oTx, oTz, oWz, oWx;  // U-stage CPML memory
    void init(int x, int z) {
        X = x; Z = z;
        for (Field<T>* f : all()) f->init(x, z);
    }
    std::vector<Field<T>*> all() {
        return {&ux, &uz, &pnx, &pnz, &snx, &snz, &ppx, &ppz, &spx, &spz, &th, &om, &qzx, &qzz,
                &qxx, &qxz, &fxx, &fzz, &fxz, &fzx, &oC, &oE, &oB, &oA, &oTx, &oTz, &oWz, &oWx};
    }
};

// Model.  With `dens` (the variable-density extension, no counterpart in the
// reference, whose equations are density-normalised, PS:373-378) the moduli
// are rho Vp^2 and rho Vs^2 and each displacement component's acceleration is
// scaled by the buoyancy 1/rho averaged onto its staggered position:
// bx(i, j) = (1/rho(i, j) + 1/rho(i+1, j)) / 2 for Ux, bz likewise along z.
template <class T>
struct Model {
    int X, Z;
    Field<T> vp, vs, ax, az;
    bool dens = false;
    Field<T> rho, bx, bz;
};

// S-stage at one cell: the four strain-like derivatives of U, the CPML
// memory of the S-stage, theta/omega and the four Q fields (PS:340-380,
// forward_s; PS:699-721, rt_s_res).  With pml=false it is reshot_s
// (PS:1001-1036): no memory terms at all.
template <class T, bool PML>
inline void s_cell(Wave<T>& w, const Model<T>& m, const T* a, int N, T dx, T dz, T dt, int i, int j,
                   T srcval) {
    const int Z = w.Z;
    const size_t c = (size_t)i * Z + j;
    const T* UX = w.ux.p() + c;
    const T* UZ = w.uz.p() + c;
    T exx = dminus(UX, (ptrdiff_t)Z, a, N, dx);   // dvxdx
    T exz = dplus(UX, (ptrdiff_t)1, a, N, dz);    // dvxdz
    T ezz = dminus(UZ, (ptrdiff_t)1, a, N, dz);   // dvzdz
    T ezx = dplus(UZ, (ptrdiff_t)Z, a, N, dx);    // dvzdx
    T vp2 = m.vp.v[c] * m.vp.v[c];
    T vs2 = m.vs.v[c] * m.vs.v[c];
    if (m.dens) {
        vp2 = vp2 * m.rho.v[c];
        vs2 = vs2 * m.rho.v[c];
    }
    if (PML) {
        T ax = m.ax.v[c], az = m.az.v[c];
        T fxx = w.fxx.v[c] = cpml(w.fxx.v[c], ax, exx, dt);
        T fzz = w.fzz.v[c] = cpml(w.fzz.v[c], az, ezz, dt);
        T fxz = w.fxz.v[c] = cpml(w.fxz.v[c], az, exz, dt);
        T fzx = w.fzx.v[c] = cpml(w.fzx.v[c], ax, ezx, dt);
        T th = vp2 * (exx + ezz - fxx - fzz);
        w.om.v[c] = vs2 * (exz - ezx - fxz + fzx);
        w.qzx.v[c] = vs2 * (ezx - fzx);
        w.qzz.v[c] = vs2 * (ezz - fzz);
        w.qxz.v[c] = vs2 * (exz - fxz);
        w.qxx.v[c] = vs2 * (exx - fxx);
        w.th.v[c] = th + srcval;   // PS:380: theta += s after the Q fields
    } else {
        T th = vp2 * (exx + ezz);
        w.om.v[c] = vs2 * (exz - ezx);
        w.qzx.v[c] = vs2 * (ezx);
        w.qzz.v[c] = vs2 * (ezz);
        w.qxz.v[c] = vs2 * (exz);
        w.qxx.v[c] = vs2 * (exx);
        w.th.v[c] = th + srcval;
    }
}

// The eight derivatives of the S-stage fields used by the U-stage
// (PS:224-279): theta_x = D+x th, theta_z = D+z th, omega_x = D-x om,
// omega_z = D-z om, A = D+z qxx, B = D-x qxz, C = D-z qzx, E = D+x qzz.
template <class T>
struct UDerivs { T tx, tz, wx, wz, A, B, C, E; };

template <class T>
inline UDerivs<T> u_derivs(const Wave<T>& w, const T* a, int N, T dx, T dz, size_t c) {
    const ptrdiff_t Z = w.Z;
    UDerivs<T> d;
    d.tx = dplus(w.th.p() + c, Z, a, N, dx);
    d.tz = dplus(w.th.p() + c, (ptrdiff_t)1, a, N, dz);
    d.wx = dminus(w.om.p() + c, Z, a, N, dx);
    d.wz = dminus(w.om.p() + c, (ptrdiff_t)1, a, N, dz);
    d.A = dplus(w.qxx.p() + c, (ptrdiff_t)1, a, N, dz);
    d.B = dminus(w.qxz.p() + c, Z, a, N, dx);
    d.C = dminus(w.qzx.p() + c, (ptrdiff_t)1, a, N, dz);
    d.E = dplus(w.qzz.p() + c, Z, a, N, dx);
    return d;
}

// U-stage with CPML (forward_u PS:281-303, rt_u_res PS:640-660): memory
// update, P/S leapfrog, level rotation, U = P + S.
template <class T>
inline void u_cell(Wave<T>& w, const Model<T>& m, const T* a, int N, T dx, T dz, T dt, int i, int j) {
    const size_t c = (size_t)i * w.Z + j;
    UDerivs<T> d = u_derivs(w, a, N, dx, dz, c);
    const T ax = m.ax.v[c], az = m.az.v[c];
    T oC = w.oC.v[c] = cpml(w.oC.v[c], az, d.C, dt);
    T oE = w.oE.v[c] = cpml(w.oE.v[c], ax, d.E, dt);
    T oB = w.oB.v[c] = cpml(w.oB.v[c], ax, d.B, dt);
    T oA = w.oA.v[c] = cpml(w.oA.v[c], az, d.A, dt);
    T oTx = w.oTx.v[c] = cpml(w.oTx.v[c], ax, d.tx, dt);
    T oTz = w.oTz.v[c] = cpml(w.oTz.v[c], az, d.tz, dt);
    T oWz = w.oWz.v[c] = cpml(w.oWz.v[c], az, d.wz, dt);
    T oWx = w.oWx.v[c] = cpml(w.oWx.v[c], ax, d.wx, dt);
    const T dt2 = dt * dt;
    T spx = d.tx - oTx + d.C - d.E - oC + oE;
    T spz = d.tz - oTz + d.B - d.A - oB + oA;
    T ssx = d.wz - oWz + d.C - d.E - oC + oE;
    T ssz = -d.wx + oWx + d.B - d.A - oB + oA;
    if (m.dens) {
        spx = spx * m.bx.v[c]; ssx = ssx * m.bx.v[c];
        spz = spz * m.bz.v[c]; ssz = ssz * m.bz.v[c];
    }
    T npx = 2 * w.pnx.v[c] - w.ppx.v[c] + dt2 * spx;
    T npz = 2 * w.pnz.v[c] - w.ppz.v[c] + dt2 * spz;
    T nsx = 2 * w.snx.v[c] - w.spx.v[c] + dt2 * ssx;
    T nsz = 2 * w.snz.v[c] - w.spz.v[c] + dt2 * ssz;
    w.ppx.v[c] = w.pnx.v[c]; w.pnx.v[c] = npx;
    w.ppz.v[c] = w.pnz.v[c]; w.pnz.v[c] = npz;
    w.spx.v[c] = w.snx.v[c]; w.snx.v[c] = nsx;
    w.spz.v[c] = w.snz.v[c]; w.snz.v[c] = nsz;
    w.ux.v[c] = npx + nsx;
    w.uz.v[c] = npz + nsz;
}

// Time-reversed U-stage without CPML (reshot_u, PS:964-979).  "prev" receives
// the value of "now" before the level shift (the reference passes d_Vpx_s
// etc. there, which the imaging condition reads afterwards).
template <class T>
inline void u_cell_reverse(Wave<T>& w, const Model<T>& m, Field<T>* prev, const T* a, int N, T dx, T dz, T dt,
                           int i, int j) {
    const size_t c = (size_t)i * w.Z + j;
    UDerivs<T> d = u_derivs(w, a, N, dx, dz, c);
    const T dt2 = dt * dt;
    T qpx = w.pnx.v[c], qpz = w.pnz.v[c], qsx = w.snx.v[c], qsz = w.snz.v[c];
    prev[0].v[c] = qpx; prev[1].v[c] = qpz; prev[2].v[c] = qsx; prev[3].v[c] = qsz;
    w.pnx.v[c] = w.ppx.v[c]; w.pnz.v[c] = w.ppz.v[c];
    w.snx.v[c] = w.spx.v[c]; w.snz.v[c] = w.spz.v[c];
    T spx = d.tx + d.C - d.E, spz = d.tz + d.B - d.A, ssx = d.wz + d.C - d.E, ssz = -d.wx + d.B - d.A;
    if (m.dens) {
        spx = spx * m.bx.v[c]; ssx = ssx * m.bx.v[c];
        spz = spz * m.bz.v[c]; ssz = ssz * m.bz.v[c];
    }
    T npx = 2 * w.pnx.v[c] - qpx + dt2 * spx;
    T npz = 2 * w.pnz.v[c] - qpz + dt2 * spz;
    T nsx = 2 * w.snx.v[c] - qsx + dt2 * ssx;
    T nsz = 2 * w.snz.v[c] - qsz + dt2 * ssz;
    w.ppx.v[c] = npx; w.ppz.v[c] = npz; w.spx.v[c] = nsx; w.spz.v[c] = nsz;
    w.ux.v[c] = npx + nsx;
    w.uz.v[c] = npz + nsz;
}

// Boundary bands (save_wavefiled PS:1230-1287; read_wavefiled1/2
// PS:1344-1424): 2N rows/columns straddling the interior edge, full length.
// The reference's buffer offsets (Q4) only shift where a value sits in its
// buffer; the set of stored cells and their values are what matters, so the
// oracle keeps one sorted list of band cells.
struct Bands {
    std::vector<int64_t> cells;
    void build(int X, int Z, int L, int N) {
        std::vector<char> in((size_t)X * Z, 0);
        for (int i = 0; i < X; ++i)
            for (int j = 0; j < Z; ++j) {
                bool b = (j >= L - N && j < L + N) || (j >= Z - L - N && j < Z - L + N) ||
                         (i >= L - N && i < L + N) || (i >= X - L - N && i < X - L + N);
                if (b) in[(size_t)i * Z + j] = 1;
            }
        cells.clear();
        for (size_t c = 0; c < in.size(); ++c)
            if (in[c]) cells.push_back((int64_t)c);
    }
};

template <class T>
struct StripStore {
    // slot-major: [slot][field 0..7][cell]; fields: ux, uz, th, om, qzx, qzz, qxx, qxz
    size_t ncell = 0;
    int nslot = 0;
    std::vector<T> data;
    void init(size_t nc, int ns) { ncell = nc; nslot = ns; data.assign((size_t)ns * 8 * nc, T(0)); }
    T* slot(int s, int f) { return data.data() + ((size_t)s * 8 + f) * ncell; }
};

template <class T>
void save_bands(Wave<T>& w, const Bands& b, StripStore<T>& st, int slot) {
    Field<T>* fs[8] = {&w.ux, &w.uz, &w.th, &w.om, &w.qzx, &w.qzz, &w.qxx, &w.qxz};
    for (int f = 0; f < 8; ++f) {
        T* dst = st.slot(slot, f);
        const T* src = fs[f]->p();
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < (int64_t)b.cells.size(); ++k) dst[k] = src[b.cells[k]];
    }
}
template <class T>
void restore_bands(Wave<T>& w, const Bands& b, StripStore<T>& st, int slot, int f0, int f1) {
    Field<T>* fs[8] = {&w.ux, &w.uz, &w.th, &w.om, &w.qzx, &w.qzz, &w.qxx, &w.qxz};
    for (int f = f0; f < f1; ++f) {
        T* dst = fs[f]->p();
        if (slot < 0) {   // level before the first step: everything was zero
#pragma omp parallel for schedule(static)
            for (int64_t k = 0; k < (int64_t)b.cells.size(); ++k) dst[b.cells[k]] = T(0);
            continue;
        }
        const T* src = st.slot(slot, f);
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < (int64_t)b.cells.size(); ++k) dst[b.cells[k]] = src[k];
    }
}

template <class T>
struct Engine {
    orc_cfg cfg;
    int X, Z, L, N;
    T a[8];
    T dx, dz, dt;
    Model<T> m;
    // FWI gradient (rtm with grad_out): rho of the formula (null: 1) and the
    // output [3][X][Z]: gradient w.r.t. Vp, w.r.t. Vs, source illumination
    const float* grad_rho = nullptr;
    T* grad_out = nullptr;

    void setup(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
               const float* rho = nullptr) {
        cfg = *c;
        X = c->X; Z = c->Z; L = c->L; N = c->N;
        for (int k = 0; k < 8; ++k) a[k] = (T)c->coeff[k];
        dx = (T)c->dx; dz = (T)c->dz; dt = (T)c->dt;
        m.X = X; m.Z = Z;
        for (Field<T>* f : {&m.vp, &m.vs, &m.ax, &m.az}) f->init(X, Z);
        for (size_t k = 0; k < (size_t)X * Z; ++k) {
            m.vp.v[k] = (T)vp[k]; m.vs.v[k] = (T)vs[k];
            m.ax.v[k] = (T)ax[k]; m.az.v[k] = (T)az[k];
        }
        m.dens = rho != nullptr;
        if (m.dens) {
            for (Field<T>* f : {&m.rho, &m.bx, &m.bz}) f->init(X, Z);
            for (int i = 0; i < X; ++i)
                for (int j = 0; j < Z; ++j) {
                    const size_t k = (size_t)i * Z + j;
                    const double b = 1.0 / rho[k];
                    const double bxn = i + 1 < X ? 1.0 / rho[k + Z] : b, bzn = j + 1 < Z ? 1.0 / rho[k + 1] : b;
                    m.rho.v[k] = (T)rho[k];
                    m.bx.v[k] = (T)(0.5 * (b + bxn));
                    m.bz.v[k] = (T)(0.5 * (b + bzn));
                }
        }
    }

    // forward_s (PS:316-384) / rt_s_res (PS:667-726) over [N, X-N) x [N, Z-N)
    void stage_s(Wave<T>& w, int t, const float* src, bool with_src) {
#pragma omp parallel for schedule(static)
        for (int i = N; i < X - N; ++i)
            for (int j = N; j < Z - N; ++j) {
                T s = T(0);
                if (with_src && i == cfg.sx && j == cfg.sz) s = (T)src[t];
                s_cell<T, true>(w, m, a, N, dx, dz, dt, i, j, s);
            }
    }
    // forward_u (PS:205-314) / rt_u_res (PS:562-665) over [N, X-N) x [N, Z-N)
    void stage_u(Wave<T>& w) {
#pragma omp parallel for schedule(static)
        for (int i = N; i < X - N; ++i)
            for (int j = N; j < Z - N; ++j) u_cell<T>(w, m, a, N, dx, dz, dt, i, j);
    }
    // FWI gradient at one back-step (the formula of the reference's unused
    // gradfun, PS:1518-1575): the source displacement U_s = P + S at the level
    // the imaging condition correlates, its four staggered derivatives, the
    // receiver's stress fields recomputed from its displacement U_r after the
    // back-step (PS:373-378; no damping memories on these cells):
    //   G_vp -= 2 rho Vp (dUx/dx + dUz/dz) theta_r
    //   G_vs -= 2 rho Vs (omega_r (dUx/dz - dUz/dx) + Qzx_r dUz/dx + Qzz_r dUz/dz
    //                     + Qxz_r dUx/dz + Qxx_r dUx/dx)
    //   S    += Ux_s^2 + Uz_s^2
    // on [L+N, X-L-N) x [L+N, Z-L-N), where every stencil reads interior
    // cells only.  The reference's dUx/dz stencil has a typo in its fourth term
    // (j - 6 for j - 3, PS:1556); the correct stencil is used.
    void gradient(const Field<T>& spx, const Field<T>& spz, const Field<T>& ssx, const Field<T>& ssz,
                  const Wave<T>& wr) {
        const size_t C = (size_t)X * Z;
        std::vector<T> usx(C), usz(C), urx(C), urz(C);
#pragma omp parallel for schedule(static)
        for (int i = L; i < X - L; ++i)
            for (int j = L; j < Z - L; ++j) {
                const size_t c = (size_t)i * Z + j;
                usx[c] = spx.v[c] + ssx.v[c]; usz[c] = spz.v[c] + ssz.v[c];
                urx[c] = wr.pnx.v[c] + wr.snx.v[c]; urz[c] = wr.pnz.v[c] + wr.snz.v[c];
            }
        T* gvp = grad_out;
        T* gvs = grad_out + C;
        T* sss = grad_out + 2 * C;
#pragma omp parallel for schedule(static)
        for (int i = L + N; i < X - L - N; ++i)
            for (int j = L + N; j < Z - L - N; ++j) {
                const size_t c = (size_t)i * Z + j;
                const ptrdiff_t sZ = Z;
                const T sxx = dminus(usx.data() + c, sZ, a, N, dx), szz = dminus(usz.data() + c, (ptrdiff_t)1, a, N, dz);
                const T szx = dplus(usz.data() + c, sZ, a, N, dx), sxz = dplus(usx.data() + c, (ptrdiff_t)1, a, N, dz);
                const T rxx = dminus(urx.data() + c, sZ, a, N, dx), rzz = dminus(urz.data() + c, (ptrdiff_t)1, a, N, dz);
                const T rzx = dplus(urz.data() + c, sZ, a, N, dx), rxz = dplus(urx.data() + c, (ptrdiff_t)1, a, N, dz);
                const T vp = m.vp.v[c], vs = m.vs.v[c], vp2 = vp * vp, vs2 = vs * vs;
                const T rho = grad_rho ? (T)grad_rho[c] : T(1);
                const T th = vp2 * (rxx + rzz), om = vs2 * (rxz - rzx);
                const T qzx = vs2 * rzx, qzz = vs2 * rzz, qxz = vs2 * rxz, qxx = vs2 * rxx;
                gvp[c] -= 2 * rho * vp * ((sxx + szz) * th);
                gvs[c] -= 2 * rho * vs * (om * (sxz - szx) + qzx * szx + qzz * szz + qxz * sxz + qxx * sxx);
                sss[c] += usx[c] * usx[c] + usz[c] * usz[c];
            }
    }

    // Receiver extraction.  The reference's test is an assignment (PS:307),
    // so every thread races to store Vx[i][Z_receive]; the deterministic
    // reading kept here is the post-update value, i.e. the one the
    // "j == Z_receive" form stores.
    void record(Wave<T>& w, T* rvx, T* rvz, int t) {
        for (int i = 0; i < X; ++i) {
            rvx[(size_t)i * cfg.nt + t] = w.ux(i, cfg.rz);
            rvz[(size_t)i * cfg.nt + t] = w.uz(i, cfg.rz);
        }
    }
    // load_record (PS:1471-1483): overwrite row Z_receive over [L, X-L)
    void inject(Wave<T>& w, const T* rvx, const T* rvz, int t) {
        for (int i = L; i < X - L; ++i) {
            w.ux(i, cfg.rz) = rvx[(size_t)i * cfg.nt + t];
            w.uz(i, cfg.rz) = rvz[(size_t)i * cfg.nt + t];
        }
    }
    // remove (PS:1634-1657): direct-wave mute, with the reference's mixed
    // float/double threshold arithmetic.
    void mute(T* rvx, T* rvz) {
        const int sx = cfg.sx, sz = cfg.sz, rz = cfg.rz;
        const float v = (float)m.vp(sx, rz);
        for (int i = 0; i < X; ++i) {
            float dist = sqrtf(float(std::abs(sx - i) * std::abs(sx - i) +
                                     std::abs(rz - sz) * std::abs(rz - sz)));
            double thr = 2 * cfg.t0 + (double)(dist * cfg.dh) * 1.0 / (double)(cfg.dt * v);
            for (int t = 0; t < cfg.nt; ++t)
                if (t < thr) {
                    rvx[(size_t)i * cfg.nt + t] = T(0);
                    rvz[(size_t)i * cfg.nt + t] = T(0);
                }
        }
    }

    // Vertical-force source (src_type 1, the extension of the library's
    // OUC_SRC_FORCE_Z; the reference only injects into theta, PS:380):
    // dt^2 w[t] is added to the P part of Uz at the source cell after the
    // leapfrog, and U = P + S there is formed again.  In float the sum is one
    // fused multiply-add, as the CUDA kernels compile it.
    void force(Wave<T>& w, const float* src, int t) {
        const int i = cfg.sx, j = cfg.sz;
        const T dt2 = dt * dt;
        T& pz = w.pnz(i, j);
        if (sizeof(T) == sizeof(float)) pz = (T)std::fma((float)dt2, (float)src[t], (float)pz);
        else pz = pz + dt2 * (T)src[t];
        w.uz(i, j) = pz + w.snz(i, j);
    }

    void forward(Wave<T>& w, const float* src, T* rvx, T* rvz, StripStore<T>* st, const Bands* b) {
        const bool theta = cfg.src_type == 0;
        for (int t = 0; t < cfg.nt; ++t) {
            stage_s(w, t, src, theta);
            stage_u(w);
            if (!theta) force(w, src, t);
            if (rvx) record(w, rvx, rvz, t);
            if (st && t != cfg.nt - 1) save_bands(w, *b, *st, t);
        }
    }

    // One RTM shot, following main()'s per-shot sequence (PS:2258-2376).
    // rec_in (X x nt, receiver-major) replaces the self-generated records if
    // given.  Outputs: images after the Laplacian (interior nx x nz), the
    // raw images and the three accumulators (padded X x Z).
    void rtm(const float* src, const float* rec_in_x, const float* rec_in_z, T* lap_pp, T* lap_ps,
             T* raw_pp, T* raw_ps, T* acc /*3*X*Z or null*/, T* rec_out /*2*X*nt or null*/,
             T* fields_out /*12*X*Z or null*/) {
        const int nt = cfg.nt;
        Wave<T> ws, wr;   // source side (forward, then reconstruction), receiver side
        ws.init(X, Z); wr.init(X, Z);
        Bands b; b.build(X, Z, L, N);
        StripStore<T> st; st.init(b.cells.size(), std::max(nt - 1, 1));
        std::vector<T> rvx((size_t)X * nt, T(0)), rvz((size_t)X * nt, T(0));
        forward(ws, src, rvx.data(), rvz.data(), &st, &b);
        if (rec_in_x) {
            for (size_t k = 0; k < rvx.size(); ++k) { rvx[k] = (T)rec_in_x[k]; rvz[k] = (T)rec_in_z[k]; }
        }
        if (cfg.do_mute) mute(rvx.data(), rvz.data());
        if (rec_out) {
            std::copy(rvx.begin(), rvx.end(), rec_out);
            std::copy(rvz.begin(), rvz.end(), rec_out + rvx.size());
        }
        // read_last_wavefiled2 (PS:2281, PS:1318-1342): the final forward state
        // seeds the reconstruction on [L-N, X-L+N)^2; the forward P/S
        // leapfrog buffers are reused in place (PS:2335).
        Wave<T>& r = ws;   // reconstruction state lives in the forward buffers
        Field<T> prev[4];  // d_Vpx_s, d_Vpz_s, d_Vsx_s, d_Vsz_s
        for (auto& f : prev) f.init(X, Z);
        {
            Field<T> keep_ux = r.ux, keep_uz = r.uz;
            Field<T> keep[6] = {r.th, r.om, r.qzx, r.qzz, r.qxx, r.qxz};
            Field<T>* dst6[6] = {&r.th, &r.om, &r.qzx, &r.qzz, &r.qxx, &r.qxz};
            r.ux.zero(); r.uz.zero();
            for (auto* f : dst6) f->zero();
            for (int i = L - N; i < X - L + N; ++i)
                for (int j = L - N; j < Z - L + N; ++j) {
                    r.ux(i, j) = keep_ux(i, j); r.uz(i, j) = keep_uz(i, j);
                    for (int f = 0; f < 6; ++f) (*dst6[f])(i, j) = keep[f](i, j);
                    prev[0](i, j) = r.pnx(i, j); prev[1](i, j) = r.pnz(i, j);
                    prev[2](i, j) = r.snx(i, j); prev[3](i, j) = r.snz(i, j);
                }
        }
        Field<T> numpp, numps, den;
        numpp.init(X, Z); numps.init(X, Z); den.init(X, Z);
        const bool src_in_band = (cfg.sz >= L - N && cfg.sz < L + N) || (cfg.sz >= Z - L - N && cfg.sz < Z - L + N) ||
                                 (cfg.sx >= L - N && cfg.sx < L + N) || (cfg.sx >= X - L - N && cfg.sx < X - L + N);
        for (int t = nt - 1; t >= 0; --t) {
            if (t < nt - 1) {
                // reshot_u (PS:2334) on the interior
#pragma omp parallel for schedule(static)
                for (int i = L; i < X - L; ++i)
                    for (int j = L; j < Z - L; ++j) u_cell_reverse<T>(r, m, prev, a, N, dx, dz, dt, i, j);
                // read_wavefiled1 (PS:2337): U strips; the reference reads slot t
                int uslot = cfg.strip_level == 0 ? t : t - 1;
                restore_bands(r, b, st, uslot, 0, 2);
                // reshot_s (PS:2340) on the interior, then read_wavefiled2 (PS:2343)
                const bool add_src = cfg.src_in_recon && !src_in_band;
#pragma omp parallel for schedule(static)
                for (int i = L; i < X - L; ++i)
                    for (int j = L; j < Z - L; ++j) {
                        T s = T(0);
                        if (add_src && i == cfg.sx && j == cfg.sz) s = (T)src[t];
                        s_cell<T, false>(r, m, a, N, dx, dz, dt, i, j, s);
                    }
                restore_bands(r, b, st, t, 2, 8);
            }
            // receiver side: load_record, rt_s_res, rt_u_res (PS:2349-2354)
            inject(wr, rvx.data(), rvz.data(), t);
            stage_s(wr, t, src, false);
            stage_u(wr);
            // corr_v (PS:2361): zero-lag PP / PS / illumination on the interior
            const Field<T>& spx = (cfg.image_align == 0 || t == nt - 1) ? prev[0] : r.pnx;
            const Field<T>& spz = (cfg.image_align == 0 || t == nt - 1) ? prev[1] : r.pnz;
            if (grad_out) {
                const Field<T>& ssx = (cfg.image_align == 0 || t == nt - 1) ? prev[2] : r.snx;
                const Field<T>& ssz = (cfg.image_align == 0 || t == nt - 1) ? prev[3] : r.snz;
                gradient(spx, spz, ssx, ssz, wr);
            }
#pragma omp parallel for schedule(static)
            for (int i = L; i < X - L; ++i)
                for (int j = L; j < Z - L; ++j) {
                    T px = spx(i, j), pz = spz(i, j);
                    numpp(i, j) += px * wr.pnx(i, j) + pz * wr.pnz(i, j);
                    den(i, j) += px * px + pz * pz;
                    numps(i, j) += px * wr.snx(i, j) + pz * wr.snz(i, j);
                }
        }
        // image_fun (PS:1441-1455) and Laplace (PS:1457-1469)
        Field<T> ipp, ips;
        ipp.init(X, Z); ips.init(X, Z);
        for (int i = L; i < X - L; ++i)
            for (int j = L; j < Z - L; ++j) {
                ipp(i, j) = numpp(i, j) / den(i, j);
                ips(i, j) = numps(i, j) / den(i, j);
            }
        const int nx = X - 2 * L, nz = Z - 2 * L;
        const T dh = (T)cfg.dx;   // main passes dx as dh (PS:2372)
        for (int i = L; i < X - L; ++i)
            for (int j = L; j < Z - L; ++j) {
                T vpp = 0, vps = 0;
                if (i >= L + 2 && i < X - L - 2 && j >= L + 2 && j < Z - L - 2) {
                    vpp = (1 / dh / dh) * (ipp(i + 1, j) + ipp(i - 1, j) - 2 * ipp(i, j) + ipp(i, j + 1) + ipp(i, j - 1) - 2 * ipp(i, j));
                    vps = (1 / dh / dh) * (ips(i + 1, j) + ips(i - 1, j) - 2 * ips(i, j) + ips(i, j + 1) + ips(i, j - 1) - 2 * ips(i, j));
                }
                size_t o = (size_t)(i - L) * nz + (j - L);
                if (lap_pp) lap_pp[o] = vpp;
                if (lap_ps) lap_ps[o] = vps;
            }
        (void)nx;
        if (raw_pp) std::copy(ipp.v.begin(), ipp.v.end(), raw_pp);
        if (raw_ps) std::copy(ips.v.begin(), ips.v.end(), raw_ps);
        if (acc) {
            size_t C = (size_t)X * Z;
            std::copy(numpp.v.begin(), numpp.v.end(), acc);
            std::copy(numps.v.begin(), numps.v.end(), acc + C);
            std::copy(den.v.begin(), den.v.end(), acc + 2 * C);
        }
        if (fields_out) dump_fields(wr, fields_out);
    }

    // RTM with the source wavefield stored during the forward pass instead of
    // reconstructed from boundary strips (the library's snapshot form): the
    // source P displacement of every K-th imaging level is kept (interior
    // only) and correlated with the receiver side there.  Imaging steps are
    // t = nt-1, nt-1-K, ...; step t uses the new level of forward step t
    // (exact alignment, and t = nt-1) or t+1 (the reference's alignment,
    // PS:964 + PS:2361).  No reconstruction, so no round-off amplification
    // by the inverse leapfrog: the reference point for long runs.
    void rtm_stored(const float* src, const float* rec_in_x, const float* rec_in_z, int K, T* lap_pp, T* lap_ps,
                    T* acc) {
        const int nt = cfg.nt, nx = X - 2 * L, nz = Z - 2 * L;
        std::vector<int> slot_of(nt, -1), slot_at(nt, -1);   // forward step -> slot, backward step -> slot
        int nslots = 0;
        for (int t = nt - 1; t >= 0; t -= K) {
            const int f = (cfg.image_align == 1 || t == nt - 1) ? t : t + 1;
            if (slot_of[f] < 0) slot_of[f] = nslots++;
            slot_at[t] = slot_of[f];
        }
        const size_t ci = (size_t)nx * nz;
        std::vector<T> store((size_t)nslots * 2 * ci);
        Wave<T> ws, wr;
        ws.init(X, Z); wr.init(X, Z);
        std::vector<T> rvx((size_t)X * nt, T(0)), rvz((size_t)X * nt, T(0));
        const bool theta = cfg.src_type == 0;
        for (int f = 0; f < nt; ++f) {
            stage_s(ws, f, src, theta);
            stage_u(ws);
            if (!theta) force(ws, src, f);
            record(ws, rvx.data(), rvz.data(), f);
            if (slot_of[f] >= 0) {
                T* d = store.data() + (size_t)slot_of[f] * 2 * ci;
#pragma omp parallel for schedule(static)
                for (int i = 0; i < nx; ++i)
                    for (int j = 0; j < nz; ++j) {
                        d[(size_t)i * nz + j] = ws.pnx(i + L, j + L);
                        d[ci + (size_t)i * nz + j] = ws.pnz(i + L, j + L);
                    }
            }
        }
        if (rec_in_x)
            for (size_t k = 0; k < rvx.size(); ++k) { rvx[k] = (T)rec_in_x[k]; rvz[k] = (T)rec_in_z[k]; }
        if (cfg.do_mute) mute(rvx.data(), rvz.data());
        Field<T> numpp, numps, den;
        numpp.init(X, Z); numps.init(X, Z); den.init(X, Z);
        for (int t = nt - 1; t >= 0; --t) {
            inject(wr, rvx.data(), rvz.data(), t);
            stage_s(wr, t, src, false);
            stage_u(wr);
            if (slot_at[t] < 0) continue;
            const T* d = store.data() + (size_t)slot_at[t] * 2 * ci;
#pragma omp parallel for schedule(static)
            for (int i = L; i < X - L; ++i)
                for (int j = L; j < Z - L; ++j) {
                    const size_t o = (size_t)(i - L) * nz + (j - L);
                    const T px = d[o], pz = d[ci + o];
                    numpp(i, j) += px * wr.pnx(i, j) + pz * wr.pnz(i, j);
                    den(i, j) += px * px + pz * pz;
                    numps(i, j) += px * wr.snx(i, j) + pz * wr.snz(i, j);
                }
        }
        const T dh = (T)cfg.dx;
        for (int i = L; i < X - L; ++i)
            for (int j = L; j < Z - L; ++j) {
                T vpp = 0, vps = 0;
                if (i >= L + 2 && i < X - L - 2 && j >= L + 2 && j < Z - L - 2) {
                    auto ip = [&](int a, int b) { return numpp(a, b) / den(a, b); };
                    auto is = [&](int a, int b) { return numps(a, b) / den(a, b); };
                    vpp = (1 / dh / dh) * (ip(i + 1, j) + ip(i - 1, j) - 2 * ip(i, j) + ip(i, j + 1) + ip(i, j - 1) - 2 * ip(i, j));
                    vps = (1 / dh / dh) * (is(i + 1, j) + is(i - 1, j) - 2 * is(i, j) + is(i, j + 1) + is(i, j - 1) - 2 * is(i, j));
                }
                const size_t o = (size_t)(i - L) * nz + (j - L);
                lap_pp[o] = vpp;
                lap_ps[o] = vps;
            }
        if (acc) {
            const size_t C = (size_t)X * Z;
            std::copy(numpp.v.begin(), numpp.v.end(), acc);
            std::copy(numps.v.begin(), numps.v.end(), acc + C);
            std::copy(den.v.begin(), den.v.end(), acc + 2 * C);
        }
    }

    // 12 fields in a fixed order: ux uz Px Pz Sx Sz th om qzx qzz qxx qxz
    static void dump_fields(Wave<T>& w, T* out) {
        Field<T>* fs[12] = {&w.ux, &w.uz, &w.pnx, &w.pnz, &w.snx, &w.snz, &w.th, &w.om, &w.qzx, &w.qzz, &w.qxx, &w.qxz};
        size_t C = (size_t)w.X * w.Z;
        for (int f = 0; f < 12; ++f) std::copy(fs[f]->v.begin(), fs[f]->v.end(), out + f * C);
    }
};

// ---- first-order velocity-stress scheme ------------------------------------
// The reference's stress (PS:487-560) and velocity (PS:390-486) kernels, which
// its main() never calls.  One step: stress (velocity derivatives -> split
// stresses with the split-field damping (1 - dt a/2) / (1 + dt a/2), source on
// theta), then velocity (stress derivatives -> P/S velocities, U = P + S,
// receiver row recorded after the update).  The damping factors and the
// update are evaluated in double precision and rounded once, as the
// reference's double literals make them; powf(v, 2) as written there.
template <class T>
struct FoWave {
    int X = 0, Z = 0;
    Field<T> vx, vz, vpx, vpz, vsx, vsz, th, om, qzx, qzz, qxx, qxz, thx, thz, omx, omz;
    void init(int x, int z) {
        X = x; Z = z;
        for (Field<T>* f : {&vx, &vz, &vpx, &vpz, &vsx, &vsz, &th, &om, &qzx, &qzz, &qxx, &qxz, &thx, &thz, &omx, &omz})
            f->init(x, z);
    }
};

inline float fo_sq(float v) { return powf(v, 2); }
inline double fo_sq(double v) { return v * v; }

template <class T>
inline T fo_damped(T a, T dt, double term, T old) {
    const double h = 0.5 * (double)dt * (double)a;
    return (T)((1.0 / (1.0 + h)) * (term + (1.0 - h) * (double)old));
}

template <class T>
inline void fo_stress_cell(FoWave<T>& w, const Model<T>& m, const T* a, int N, T dx, T dz, T dt, int i, int j,
                           T srcval) {
    const int Z = w.Z;
    const size_t c = (size_t)i * Z + j;
    const T exx = dminus(w.vx.p() + c, (ptrdiff_t)Z, a, N, dx);   // dvxdx
    const T exz = dplus(w.vx.p() + c, (ptrdiff_t)1, a, N, dz);    // dvxdz
    const T ezz = dminus(w.vz.p() + c, (ptrdiff_t)1, a, N, dz);   // dvzdz
    const T ezx = dplus(w.vz.p() + c, (ptrdiff_t)Z, a, N, dx);    // dvzdx
    const T vp2 = fo_sq(m.vp.v[c]), vs2 = fo_sq(m.vs.v[c]);
    const T ax = m.ax.v[c], az = m.az.v[c];
    w.thx.v[c] = fo_damped(ax, dt, (double)(dt * vp2 * exx), w.thx.v[c]);
    w.thz.v[c] = fo_damped(az, dt, (double)(dt * vp2 * ezz), w.thz.v[c]);
    w.omx.v[c] = fo_damped(ax, dt, (double)(-dt * vs2 * ezx), w.omx.v[c]);
    w.omz.v[c] = fo_damped(az, dt, (double)(dt * vs2 * exz), w.omz.v[c]);
    w.qxx.v[c] = fo_damped(ax, dt, (double)(dt * vs2 * exx), w.qxx.v[c]);
    w.qxz.v[c] = fo_damped(az, dt, (double)(dt * vs2 * exz), w.qxz.v[c]);
    w.qzx.v[c] = fo_damped(ax, dt, (double)(dt * vs2 * ezx), w.qzx.v[c]);
    w.qzz.v[c] = fo_damped(az, dt, (double)(dt * vs2 * ezz), w.qzz.v[c]);
    w.th.v[c] = w.thx.v[c] + w.thz.v[c] + srcval;
    w.om.v[c] = w.omx.v[c] + w.omz.v[c];
}

template <class T>
inline void fo_velocity_cell(FoWave<T>& w, const Model<T>& m, const T* a, int N, T dx, T dz, T dt, int i, int j) {
    const ptrdiff_t Z = w.Z;
    const size_t c = (size_t)i * Z + j;
    const T tx = dplus(w.th.p() + c, Z, a, N, dx), tz = dplus(w.th.p() + c, (ptrdiff_t)1, a, N, dz);
    const T wx = dminus(w.om.p() + c, Z, a, N, dx), wz = dminus(w.om.p() + c, (ptrdiff_t)1, a, N, dz);
    const T dux_xdz = dplus(w.qxx.p() + c, (ptrdiff_t)1, a, N, dz);
    const T dux_zdx = dminus(w.qxz.p() + c, Z, a, N, dx);
    const T duz_xdz = dminus(w.qzx.p() + c, (ptrdiff_t)1, a, N, dz);
    const T duz_zdx = dplus(w.qzz.p() + c, Z, a, N, dx);
    const T ax = m.ax.v[c], az = m.az.v[c];
    auto upd = [&](T damp, T old, T sum) {
        const double h = 0.5 * (double)dt * (double)damp;
        return (T)((1.0 / (1.0 + h)) * ((1 - h) * (double)old + (double)(dt * sum)));
    };
    w.vpx.v[c] = upd(ax, w.vpx.v[c], tx + duz_xdz - duz_zdx);
    w.vpz.v[c] = upd(az, w.vpz.v[c], tz + dux_zdx - dux_xdz);
    w.vsx.v[c] = upd(ax, w.vsx.v[c], wz + duz_xdz - duz_zdx);
    w.vsz.v[c] = upd(az, w.vsz.v[c], -wx + dux_zdx - dux_xdz);
    w.vx.v[c] = w.vpx.v[c] + w.vsx.v[c];
    w.vz.v[c] = w.vpz.v[c] + w.vsz.v[c];
}

template <class T>
int run_forward_fo(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                   const float* src, T* rec_vx, T* rec_vz, T* fields_out) {
    Engine<T> e;
    e.setup(c, vp, vs, ax, az);
    const int X = c->X, Z = c->Z, N = c->N, nt = c->nt;
    FoWave<T> w;
    w.init(X, Z);
    for (int t = 0; t < nt; ++t) {
#pragma omp parallel for schedule(static)
        for (int i = N; i < X - N; ++i)
            for (int j = N; j < Z - N; ++j) {
                const T s = (i == c->sx && j == c->sz) ? (T)src[t] : T(0);
                fo_stress_cell<T>(w, e.m, e.a, N, e.dx, e.dz, e.dt, i, j, s);
            }
#pragma omp parallel for schedule(static)
        for (int i = N; i < X - N; ++i)
            for (int j = N; j < Z - N; ++j) fo_velocity_cell<T>(w, e.m, e.a, N, e.dx, e.dz, e.dt, i, j);
        for (int i = 0; i < X; ++i) {
            if (rec_vx) rec_vx[(size_t)i * nt + t] = w.vx(i, c->rz);
            if (rec_vz) rec_vz[(size_t)i * nt + t] = w.vz(i, c->rz);
        }
    }
    if (fields_out) {
        Field<T>* fs[16] = {&w.vx, &w.vz, &w.vpx, &w.vpz, &w.vsx, &w.vsz, &w.th, &w.om,
                            &w.qzx, &w.qzz, &w.qxx, &w.qxz, &w.thx, &w.thz, &w.omx, &w.omz};
        const size_t C = (size_t)X * Z;
        for (int k = 0; k < 16; ++k) std::copy(fs[k]->v.begin(), fs[k]->v.end(), fields_out + k * C);
    }
    return 0;
}

// First-order receiver back-propagation: the reference's
// stress_backward_propagation (PS:821-887) and velocity_backward_propagation
// (PS:728-820) are the stress/velocity updates without source and record;
// before each step (t = nt-1 .. 0) the receiver row of U is replaced by the
// records on [L, X-L), as load_record (PS:1472-1481) does in the launched
// receiver path (PS:2319).  rec_*: X x nt.
template <class T>
int run_backward_fo(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                    const float* rec_vx, const float* rec_vz, T* fields_out) {
    Engine<T> e;
    e.setup(c, vp, vs, ax, az);
    const int X = c->X, Z = c->Z, N = c->N, L = c->L, nt = c->nt;
    FoWave<T> w;
    w.init(X, Z);
    for (int t = nt - 1; t >= 0; --t) {
        for (int i = L; i < X - L; ++i) {
            w.vx(i, c->rz) = (T)rec_vx[(size_t)i * nt + t];
            w.vz(i, c->rz) = (T)rec_vz[(size_t)i * nt + t];
        }
#pragma omp parallel for schedule(static)
        for (int i = N; i < X - N; ++i)
            for (int j = N; j < Z - N; ++j) fo_stress_cell<T>(w, e.m, e.a, N, e.dx, e.dz, e.dt, i, j, T(0));
#pragma omp parallel for schedule(static)
        for (int i = N; i < X - N; ++i)
            for (int j = N; j < Z - N; ++j) fo_velocity_cell<T>(w, e.m, e.a, N, e.dx, e.dz, e.dt, i, j);
    }
    if (fields_out) {
        Field<T>* fs[16] = {&w.vx, &w.vz, &w.vpx, &w.vpz, &w.vsx, &w.vsz, &w.th, &w.om,
                            &w.qzx, &w.qzz, &w.qxx, &w.qxz, &w.thx, &w.thz, &w.omx, &w.omz};
        const size_t C = (size_t)X * Z;
        for (int k = 0; k < 16; ++k) std::copy(fs[k]->v.begin(), fs[k]->v.end(), fields_out + k * C);
    }
    return 0;
}

template <class T>
int run_forward(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                const float* src, T* rec_vx, T* rec_vz, T* fields_out, const float* rho = nullptr) {
    Engine<T> e;
    e.setup(c, vp, vs, ax, az, rho);
    Wave<T> w;
    w.init(c->X, c->Z);
    std::vector<T> rx((size_t)c->X * c->nt), rz((size_t)c->X * c->nt);
    e.forward(w, src, rx.data(), rz.data(), nullptr, nullptr);
    if (rec_vx) std::copy(rx.begin(), rx.end(), rec_vx);
    if (rec_vz) std::copy(rz.begin(), rz.end(), rec_vz);
    if (fields_out) Engine<T>::dump_fields(w, fields_out);
    return 0;
}

}  // namespace

extern "C" {

int orc_forward_f32(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                    const float* src, float* rec_vx, float* rec_vz, float* fields_out) {
    return run_forward<float>(c, vp, vs, ax, az, src, rec_vx, rec_vz, fields_out);
}
int orc_forward_f64(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                    const float* src, double* rec_vx, double* rec_vz, double* fields_out) {
    return run_forward<double>(c, vp, vs, ax, az, src, rec_vx, rec_vz, fields_out);
}
int orc_rtm_f32(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                const float* src, const float* rec_x, const float* rec_z, float* lap_pp, float* lap_ps,
                float* raw_pp, float* raw_ps, float* acc, float* rec_out, float* fields_out) {
    Engine<float> e;
    e.setup(c, vp, vs, ax, az);
    e.rtm(src, rec_x, rec_z, lap_pp, lap_ps, raw_pp, raw_ps, acc, rec_out, fields_out);
    return 0;
}
int orc_rtm_f64(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                const float* src, const float* rec_x, const float* rec_z, double* lap_pp, double* lap_ps,
                double* raw_pp, double* raw_ps, double* acc, double* rec_out, double* fields_out) {
    Engine<double> e;
    e.setup(c, vp, vs, ax, az);
    e.rtm(src, rec_x, rec_z, lap_pp, lap_ps, raw_pp, raw_ps, acc, rec_out, fields_out);
    return 0;
}

// RTM from the stored source wavefield (Engine::rtm_stored), every K-th
// imaging level, in double precision: the FP64 reference of the snapshot form.
int orc_rtm_stored_f64(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                       const float* src, const float* rec_x, const float* rec_z, int K, double* lap_pp,
                       double* lap_ps, double* acc) {
    if (K < 1) return 1;
    Engine<double> e;
    e.setup(c, vp, vs, ax, az);
    e.rtm_stored(src, rec_x, rec_z, K, lap_pp, lap_ps, acc);
    return 0;
}

// RTM with the FWI gradient (see Engine::gradient): grad [3][X][Z] receives
// the gradient w.r.t. Vp, w.r.t. Vs and the source illumination of one shot;
// rho (padded, may be NULL for 1) enters the gradient formula only.
int orc_rtm_grad_f64(const orc_cfg* c, const float* vp, const float* vs, const float* rho, const float* ax,
                     const float* az, const float* src, const float* rec_x, const float* rec_z, double* lap_pp,
                     double* lap_ps, double* grad) {
    Engine<double> e;
    e.setup(c, vp, vs, ax, az);
    e.grad_rho = rho;
    std::fill(grad, grad + 3 * (size_t)c->X * c->Z, 0.0);
    e.grad_out = grad;
    e.rtm(src, rec_x, rec_z, lap_pp, lap_ps, nullptr, nullptr, nullptr, nullptr, nullptr);
    return 0;
}
int orc_rtm_grad_f32(const orc_cfg* c, const float* vp, const float* vs, const float* rho, const float* ax,
                     const float* az, const float* src, const float* rec_x, const float* rec_z, float* lap_pp,
                     float* lap_ps, float* grad) {
    Engine<float> e;
    e.setup(c, vp, vs, ax, az);
    e.grad_rho = rho;
    std::fill(grad, grad + 3 * (size_t)c->X * c->Z, 0.f);
    e.grad_out = grad;
    e.rtm(src, rec_x, rec_z, lap_pp, lap_ps, nullptr, nullptr, nullptr, nullptr, nullptr);
    return 0;
}

// First-order velocity-stress forward modeling (see run_forward_fo):
// records X x nt, fields 16 x X x Z (Vx Vz Vpx Vpz Vsx Vsz theta omega Qzx
// Qzz Qxx Qxz theta_x theta_z omega_x omega_z).
int orc_forward_fo_f32(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                       const float* src, float* rec_vx, float* rec_vz, float* fields_out) {
    return run_forward_fo<float>(c, vp, vs, ax, az, src, rec_vx, rec_vz, fields_out);
}
int orc_forward_fo_f64(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                       const float* src, double* rec_vx, double* rec_vz, double* fields_out) {
    return run_forward_fo<double>(c, vp, vs, ax, az, src, rec_vx, rec_vz, fields_out);
}
// First-order receiver back-propagation (see run_backward_fo).
int orc_backward_fo_f32(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                        const float* rec_vx, const float* rec_vz, float* fields_out) {
    return run_backward_fo<float>(c, vp, vs, ax, az, rec_vx, rec_vz, fields_out);
}
int orc_backward_fo_f64(const orc_cfg* c, const float* vp, const float* vs, const float* ax, const float* az,
                        const float* rec_vx, const float* rec_vz, double* fields_out) {
    return run_backward_fo<double>(c, vp, vs, ax, az, rec_vx, rec_vz, fields_out);
}

// Variable-density variants (rho: padded X x Z density; see Model).
int orc_forward_rho_f64(const orc_cfg* c, const float* vp, const float* vs, const float* rho, const float* ax,
                        const float* az, const float* src, double* rec_vx, double* rec_vz, double* fields_out) {
    return run_forward<double>(c, vp, vs, ax, az, src, rec_vx, rec_vz, fields_out, rho);
}
int orc_rtm_rho_f64(const orc_cfg* c, const float* vp, const float* vs, const float* rho, const float* ax,
                    const float* az, const float* src, const float* rec_x, const float* rec_z, double* lap_pp,
                    double* lap_ps, double* raw_pp, double* raw_ps, double* acc, double* rec_out, double* fields_out) {
    Engine<double> e;
    e.setup(c, vp, vs, ax, az, rho);
    e.rtm(src, rec_x, rec_z, lap_pp, lap_ps, raw_pp, raw_ps, acc, rec_out, fields_out);
    return 0;
}

// Edge padding of an interior model into the absorbing layer (xiangbian,
// PS:37-119): sides copy the nearest interior row/column, corners the
// nearest interior corner cell.  In place on a padded X x Z array.
void orc_pad_model(float* f, int X, int Z, int L) {
    auto at = [&](int i, int j) -> float& { return f[(size_t)i * Z + j]; };
    for (int i = L; i < X - L; ++i) {
        for (int j = 0; j < L; ++j) at(i, j) = at(i, L);
        for (int j = Z - L; j < Z; ++j) at(i, j) = at(i, Z - L - 1);
    }
    for (int j = L; j < Z - L; ++j) {
        for (int i = 0; i < L; ++i) at(i, j) = at(L, j);
        for (int i = X - L; i < X; ++i) at(i, j) = at(X - L - 1, j);
    }
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Z; ++j) {
            bool cx = i < L || i >= X - L, cz = j < L || j >= Z - L;
            if (cx && cz) at(i, j) = at(i < L ? L : X - L - 1, j < L ? L : Z - L - 1);
        }
}

// Damping profile (PS:2067-2105): d = log10(1/R) * 1.5 * Vp / L * (dist/L)^4
// with L in grid points; the left/top layers have L damped cells, the
// right/bottom ones L-1 (strict ">" at PS:2077).
void orc_cpml_profile(const float* vp, int X, int Z, int L, double R, float* ax, float* az) {
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Z; ++j) {
            size_t c = (size_t)i * Z + j;
            double v = vp[c];
            if (i < L) ax[c] = (float)(log10(1.0 / R) * 1.5 * v / L * pow(1.0 * (L - i) / L, 4.0));
            else if (i > X - L) ax[c] = (float)(log10(1.0 / R) * 1.5 * v / L * pow(1.0 * (i - X + L) / L, 4.0));
            else ax[c] = 0.0f;
            if (j < L) az[c] = (float)(log10(1.0 / R) * 1.5 * v / L * pow(1.0 * (L - j) / L, 4.0));
            else if (j > Z - L) az[c] = (float)(log10(1.0 / R) * 1.5 * v / L * pow(1.0 * (j - Z + L) / L, 4.0));
            else az[c] = 0.0f;
        }
}

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// Ricker wavelet as the reference's main() builds it (PS:1954-1958):
// Nk = PI^2 FM^2 dt^2 formed in double from PI = 3.1415926 (PS:14) and
// stored as float, t0 = ceil(1 / (FM dt)) samples, the exponent taken in
// float, the product in double and stored as float.
int orc_ricker(float fm, float dt, int nt, float* out, int* t0_out) {
    if (!(fm > 0) || !(dt > 0) || nt < 1 || !out) return 1;
    const double pi_ref = 3.1415926;
    const double f = fm;
    const float nk = (float)(pi_ref * pi_ref * f * f * dt * dt);
    const int t0 = (int)ceil(1.0 / (f * dt));
    for (int t = 0; t < nt; ++t) {
        const int d = t - t0;
        const float e = std::exp(-nk * d * d);
        out[t] = (float)((1.0 - 2.0 * nk * d * d) * e);
    }
    if (t0_out) *t0_out = t0;
    return 0;
}

}  // extern "C"
