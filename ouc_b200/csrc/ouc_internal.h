// Internal definitions shared by the kernels and the host orchestration.
//
// Device layout ("pitched padded grid").  Every cell field lives in its own
// allocation of (Xc + 2*GX) rows by `pitch` floats:
//   - Xc = X rounded up to the tile height, Zc = Z rounded up to the tile
//     width, so a tile never needs a bounds test on its own cells;
//   - GX guard rows above and below and ZOFF guard columns left of column 0
//     (and at least ZOFF right of Zc), all zero and never written, so the
//     halo loads of a tile at the grid edge stay inside the allocation;
//   - `pitch` is a multiple of 32 floats, so every row starts on a 128-byte
//     boundary and a float4 at a column multiple of 4 is 16-byte aligned.
// Field pointers passed to kernels point at cell (0, 0): element (i, j) is
// f[i * pitch + j] for i in [-GX, Xc+GX) and j in [-ZOFF, Zc+ZOFF).
#pragma once
#include <cuda.h>            // CUtensorMap (the type; its encoder is reached through the runtime)
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ouc {

constexpr int kGX = 16;        // guard rows on each side
constexpr int kZOFF = 16;      // guard columns on each side
constexpr int kThreads = 256;  // threads per step CTA

// Tile grids of the step kernels (32 x 64 cell tiles).  The forward and
// receiver steps tile the padded grid from (0, 0).  The reconstruction
// updates only the interior [L, X-L) x [L, Z-L), so its tiles start at
// x = L and z = L rounded down to a multiple of 4 (float4 alignment): at
// 1000 x 500 with L = 30 that is 32 x 8 tiles instead of the 33 x 9 that
// tiles from the origin would need.  Xc x Zc is the extent the field
// allocations hold (before their guard rows and columns) so that every
// tile's cells lie inside.
struct TileGrid {
    int tiles_x, tiles_z;          // full step, from (0, 0)
    int rec_x0, rec_z0;            // reconstruction: cell origin of its first tile
    int rec_tiles_x, rec_tiles_z;
    int Xc, Zc;
};
inline int rec_tiles_for(int X, int L) { return (X - 2 * L + 31) / 32; }
inline TileGrid tile_grid(int X, int Z, int L) {
    TileGrid g;
    g.tiles_x = (X + 31) / 32;
    g.tiles_z = (Z + 63) / 64;
    g.rec_x0 = L;
    g.rec_z0 = L & ~3;
    g.rec_tiles_x = rec_tiles_for(X, L);
    g.rec_tiles_z = (Z - L - g.rec_z0 + 63) / 64;
    g.Xc = g.tiles_x * 32 > g.rec_x0 + g.rec_tiles_x * 32 ? g.tiles_x * 32 : g.rec_x0 + g.rec_tiles_x * 32;
    g.Zc = g.tiles_z * 64 > g.rec_z0 + g.rec_tiles_z * 64 ? g.tiles_z * 64 : g.rec_z0 + g.rec_tiles_z * 64;
    return g;
}

// Float32 staggered weights a_1..a_N by half-order N (row N).  N = 6: the
// reference's literals (PS:221).  Other N: the exact Taylor solution of
// sum_k c_k (2k-1)^(2n-1) = [n==1], rounded to float32 where used.  The one
// table every entry point takes its stencil from.
inline constexpr double kStencilWeights[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0, 0, 0, 0, 0, 0},
    {1.125, -1.0 / 24.0, 0, 0, 0, 0},
    {75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0, 0, 0},
    {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0, 0, 0},
    {19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0, 0},
    {1.2213364, -9.6931458e-2, 1.7447662e-2, -2.9672895e-3, 3.5900540e-4, -2.1847812e-5},
};

enum Mode : int { kFwd = 0, kRcv = 1, kRec = 2 };

// Boundary ring: the cells within N of the interior edge, on both sides
// (the reference's four strips of 2N rows/columns, PS:1230-1287, trimmed to
// the box [L-N, X-L+N) x [L-N, Z-L+N) that the reconstruction reads).
struct Ring {
    int L, N, X, Z;
    int W, H;   // box extent along x and z: nx + 2N, nz + 2N
    int R;      // ring cells
    __host__ __device__ static Ring make(int X, int Z, int L, int N) {
        Ring r;
        r.L = L; r.N = N; r.X = X; r.Z = Z;
        r.W = X - 2 * L + 2 * N;
        r.H = Z - 2 * L + 2 * N;
        r.R = 4 * N * r.W + 4 * N * (r.H - 4 * N);
        return r;
    }
    // Index of cell (i, j) in the ring, or -1 when the cell is not in it.
    // Order: top band (j near the top interior edge) W x 2N, bottom band
    // W x 2N, left band 2N x (H-4N), right band 2N x (H-4N); z contiguous.
    __host__ __device__ __forceinline__ int index(int i, int j) const {
        const int ii = i - (L - N), jj = j - (L - N);
        if (ii < 0 || ii >= W || jj < 0 || jj >= H) return -1;
        const int n2 = 2 * N;
        if (jj < n2) return ii * n2 + jj;
        if (jj >= H - n2) return W * n2 + ii * n2 + (jj - (H - n2));
        const int hm = H - 2 * n2;
        if (ii < n2) return 2 * W * n2 + ii * hm + (jj - n2);
        if (ii >= W - n2) return 2 * W * n2 + n2 * hm + (ii - (W - n2)) * hm + (jj - n2);
        return -1;
    }
    __host__ __device__ __forceinline__ bool in_box(int i, int j) const {
        return i >= L - N && i < X - L + N && j >= L - N && j < Z - L + N;
    }
};

// Strip slot layout: [slot][field][ring cell], fields in the order
// Ux, Uz, theta, omega, Qzx, Qzz, Qxx, Qxz.
enum StripField : int { kSUx = 0, kSUz, kSTh, kSOm, kSQzx, kSQzz, kSQxx, kSQxz, kStripFields };

// Storage of the boundary strips (ouc_config.strip_precision).
//   kStripF32:  float, as computed;
//   kStripF16:  IEEE half of v * 2^k, one power-of-two scale k per slot and
//               field, chosen from that slot's largest |v| so that it maps
//               into [2^14, 2^15); the forward step writes float values to a
//               two-slot staging ring and reduces their maxima, and the next
//               step (or k_strip_pack after the last one) converts the slot
//               once its maxima are complete;
//   kStripBF16: bfloat16 of v (float's exponent range: no scale).
enum StripPrec : int { kStripF32 = 0, kStripF16 = 1, kStripBF16 = 2 };

__host__ __device__ constexpr int strip_elem_bytes(int prec) { return prec == kStripF32 ? 4 : 2; }

// Per-shot constants of a batch (uploaded once per batch).
struct ShotDesc {
    int sx, sz, rz, src_type;      // padded coordinates
    const float* wavelet;          // nt samples
    float* gather_x;               // time-major gathers [nt][X]
    float* gather_z;
    void* strips;                  // [slot][8 fields][ring] of the strip element type, or null
    float* stage;                  // kStripF16: staging ring [2][8 fields][ring] floats
    unsigned* amax;                // kStripF16: [slot][8 fields] bits of the largest |v| (float)
    // Geometry of this shot's grid.  Shots of one launch share Z, L, N and
    // the pitch but may differ in width (per-shot sub-grids of a survey); a
    // CTA whose tile lies beyond its shot's width exits at once.
    int X;                         // padded width (rows along x)
    int tiles_x;                   // tile rows of the full step
    int rec_tiles_x;               // tile rows of the reconstruction (interior)
    Ring ring;                     // boundary ring of this grid
    size_t off;                    // offset (floats) of this shot's fields from shot 0's: b * shot_stride
                                   // for shot b of a launch (the tensor copies address slot b)
    size_t strip_slot;             // floats per strip slot
    const float* vp2;              // model views of this grid, cell (0, 0): the moduli
    const float* vs2;              // (rho) Vp^2 and (rho) Vs^2, damping x and z,
    const float* ax;
    const float* az;
    const float* bx;               // and with StepArgs.density the buoyancy at the Ux
    const float* bz;               // and Uz positions
};

struct StepArgs {
    // 4-D tensor map of the state block (columns of the pitch, rows with the
    // guard rows, field, shot slot) whose box is one tile's U box (UC x UR
    // of TileGeo<N>): the step kernels bring the U box into shared memory
    // with one cp.async.bulk.tensor per field.  state0 is the block's start
    // (field 0 of slot 0, guard row and column 0); launch_step refuses a
    // launch whose map is missing or whose now[] fields are not fields of
    // the block, and fills now_field from now[].
    alignas(64) CUtensorMap box_map;
    alignas(64) CUtensorMap own_map;     // the same block, box = one tile's own cells (TZ x TX): L2 prefetches
    alignas(64) CUtensorMap s_map;       // the same block, box = one tile's S region (SC x SR): L2 prefetches
    const float* state0;
    size_t fstride;                   // floats per field of the block
    int nfields;                      // fields per shot slot of the block
    int now_field[4];                 // field index of now[0..3]
    int past_field[4], rcv_field[4], acc_field[3];   // field indices of past, rcv, acc (-1: not in the block)
    int o_field[8], fold_field[4];                   // and of the U- and S-stage CPML memories
    unsigned copy_tx_extra;           // test hook: bytes expected beyond the copies (0; ouc_debug_copy_stall)
    int X, Z, pitch, L;
    int tiles_z, tile_x0, tile_z0;    // tile columns of this launch; cell origin of its first tile
    int t;                            // time step index
    int slot_u, slot_s;               // kRec: strip slots holding U and theta..Qxz at level t+1
    int record, save;                 // kFwd: write gathers / boundary strips this step
    int src_recon;                    // kRec: add the source term at (sx, sz) outside the ring
    int img_past;                     // kRec: correlate with level t+2 (reference alignment)
    int strip_prec;                   // StripPrec of the strips
    int comp_image;                   // kRec: compensated (Kahan) imaging sums, comp[] below
    int density;                      // variable density: scale the U-stage by the buoyancy
    int seg_rows;                     // > 0: the x-marching kernel, segments of this many rows (a multiple of 16);
                                      // 0: one CTA per 32 x 64 tile; -1: the tile kernel with a dynamic queue
    int nsm;                          // SMs of the device (persistent grid of the queue form)
    int* queue;                       // queue form: [mode][claim counter, finished CTAs], zero between launches
    const int* order[2];              // queue form: tiles (tx << 16 | tz), heaviest first: full grid, reconstruction
    int* err;                         // device word: kernels record OUC_ETIMEOUT-class failures here (or null)
    float a[6];                       // stencil weights a_1..a_N
    float dx, dz, dt, dt2;
    float rdx, rdz;                   // RN(1/dx), RN(1/dz)
    // Fields of shot 0; shot b adds b * shot_stride floats.
    // leapfrog state: now (level n, read with halo), past (level n-1, read
    // at own cells, overwritten with level n+1)
    const float* now[4];              // Px Pz Sx Sz
    float* past[4];
    // S-stage CPML memory, ping-pong: read old (halo), write new (own)
    const float* f_old[4];            // xx zz xz zx
    float* f_new[4];
    // U-stage CPML memory, in place at own cells
    float* o[8];                      // C E B A Tx Tz Wz Wx
    // kRec imaging
    const float* rcv[4];              // receiver Px Pz Sx Sz after this back-step
    float* acc[3];                    // PP, PS, illumination accumulators
    float* comp[3];                   // their compensation terms (comp_image)
    // uniform geometry of the batch, for the kernels other than k_step
    // (k_step reads each shot's geometry from its ShotDesc)
    const float* vp2;
    const float* vs2;
    const float* ax;
    const float* az;
    size_t shot_stride;               // floats between consecutive shots' state
    size_t strip_slot;                // floats per strip slot
    Ring ring;
    const ShotDesc* shots;            // device array indexed by blockIdx.y
};

struct FinalizeArgs {
    int X, Z, pitch, L;
    int nshots;
    size_t shot_stride;    // between shots' accumulators (floats)
    float dh;
    const float* acc[3];   // shot 0
    const float* comp[3];  // compensation terms of the accumulators, or null (plain sums)
    float* img;            // [shot][2][nx][nz] dense, or null
    double* stack[3];      // nx*nz dense FP64: PP, PS, illumination (or null)
    double illum_scale;    // illumination into the stack x this (imaged levels: every K-th)
    const int* status;     // device status word (or null): nonzero leaves the stack untouched
};

// Source-wavefield snapshots (ouc_config.snapshot_every = K >= 1): the
// source P displacement (Px, Pz) on the interior at every K-th imaging level,
// stored as [shot][slot][2][nx][nz] elements of the strip type (StripPrec),
// f16 scaled by 2^k per slot and component (k from that snapshot's largest
// |v|, as for the strips).  The backward pass images those levels only.
struct SnapArgs {
    int X, Z, pitch, L, nx, nz;
    size_t shot_stride;      // state floats between shots
    int prec;                // StripPrec of the snapshots
    int slot;
    size_t shot_elems;       // snapshot elements per shot (all slots)
    void* snaps;             // shot 0, slot 0
    unsigned* amax;          // f16: [shot][slot][2] bits of the largest |v|
    int nslots;
    // pack: the source P level to store (shot 0, pitched)
    const float* px;
    const float* pz;
    // imaging: receiver fields after the back-step, accumulators (shot 0)
    const float* rcv[4];
    float* acc[3];
    float* comp[3];
    int comp_image;
};

// FWI gradient of one back-step (see k_grad).
struct GradArgs {
    int X, Z, pitch, L, N;
    int nshots;
    float a[6];
    float dx, dz;
    const float* src[4];     // source Px Pz Sx Sz at the imaged level (shot 0)
    const float* rcv[4];     // receiver Px Pz Sx Sz after the back-step (shot 0)
    size_t shot_stride;      // state floats between shots
    const float* vp;         // Vp, Vs and (or null: 1) rho of the formula
    const float* vs;
    const float* rho;
    float* g[3];             // shot 0: gradient w.r.t. Vp, w.r.t. Vs, source illumination
    size_t grad_stride;      // floats between shots' gradient accumulators
};
struct GradStackArgs {
    int X, Z, pitch, L, nshots;
    const float* g[3];
    size_t grad_stride;
    double* stack[3];        // nx*nz dense FP64
};

// Host-side launchers (kernels.cu)
// Encode StepArgs::box_map for a state block at `state0` (nslots shot slots
// of nfields fields of rows x pitch floats each) and half-order N.
cudaError_t encode_box_map(StepArgs& a, const float* state0, int pitch, int rows, int nfields, int nslots,
                           size_t fstride, int N);
int launch_step(int N, Mode mode, const StepArgs& a, int tiles_x, int nshots, cudaStream_t s);
// Segments of the x-marching kernel for a launch (rows of the widest shot).
int march_segments(Mode mode, const StepArgs& a);
cudaError_t configure_step_kernels(int N);
int step_smem_bytes(int N);
void launch_image_only(const StepArgs& a, int nshots, cudaStream_t s);
void launch_finalize(const FinalizeArgs& f, cudaStream_t s);
void launch_mute(float* gx, float* gz, int X, int nt, int sx, int sz, int rz, int t0, float dt, float dh, float v,
                 cudaStream_t s);
void launch_transpose(const float* in, float* out, int rows, int cols, cudaStream_t s);
// Bit 1 of *status when any of n floats (16-byte aligned) is not finite.
void launch_finite_check(const float* p, size_t n, int* status, cudaStream_t s);
void launch_pack_fields(const float* const* f, int nf, int X, int Z, int pitch, float* out, cudaStream_t s);
void launch_strip_pack(const ShotDesc* shots, int nshots, int slot, int ring, size_t strip_slot, cudaStream_t s);
void launch_snap_store(const SnapArgs& a, int nshots, cudaStream_t s);
void launch_image_snap(const SnapArgs& a, int nshots, cudaStream_t s);
void launch_grad(const GradArgs& a, cudaStream_t s);
void launch_grad_stack(const GradStackArgs& a, cudaStream_t s);

}  // namespace ouc
