// Private: the context object behind the C ABI and the host-side step
// helpers that api.cu implements, shared with the learned-corrector driver
// (learned.cu).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/ouc.h"
#include "ouc_internal.h"

namespace ouc {
constexpr int kFieldsPerSide = 24;                    // now 4, past 4, F old 4, F new 4, O 8
constexpr int kFieldsPerShot = 2 * kFieldsPerSide + 6;   // source side, receiver side, accumulators + compensation

// Field pointers of one wavefield (shot 0 of the batch).
struct Side {
    float* now[4];
    float* past[4];
    float* fo[4];
    float* fn[4];
    float* o[8];
    void swap_levels() { for (int k = 0; k < 4; ++k) std::swap(now[k], past[k]); }
    void swap_memory() { for (int k = 0; k < 4; ++k) std::swap(fo[k], fn[k]); }
};

}  // namespace ouc

struct ouc_ctx {
    using Ring = ouc::Ring;
    using Side = ouc::Side;
    using ShotDesc = ouc::ShotDesc;
    using StepArgs = ouc::StepArgs;
    static constexpr int kGX = ouc::kGX, kZOFF = ouc::kZOFF;
    ouc_config cfg;
    int X = 0, Z = 0, L = 0, N = 0, nx = 0, nz = 0, nt = 0;
    int Xc = 0, Zc = 0, pitch = 0;
    int batch = 1;               // shots the device state holds (cfg.max_batch)
    int run_batch = 1;           // shots advanced per launch (<= batch; ouc_tune_batch)
    int seg_rows = 0;            // step kernel: x-marching segments of this many rows, or 0 for 32 x 64 tiles
    bool copy_stall = false;     // test hook (ouc_debug_copy_stall): tile copy waits run out
    int* d_status = nullptr;     // device status word: bit 0 a copy wait timed out, bit 1 a non-finite field
    int nsm = 148;               // SMs of the device
    int* d_queue = nullptr;      // dynamic-queue form: [mode][claim counter, finished CTAs]
    int* d_order[2] = {nullptr, nullptr};   // its tile orders, heaviest first: full grid, reconstruction
    size_t fstride = 0;          // floats per field allocation
    alignas(64) CUtensorMap box_map;   // tensor map of the state block (StepArgs::box_map)
    alignas(64) CUtensorMap own_map;   // and its own-cell box form (StepArgs::own_map)
    alignas(64) CUtensorMap s_map;     // and its S-region box form (StepArgs::s_map)
    const float* box_state0 = nullptr;  // its start (null until encoded)
    size_t shot_stride = 0;      // floats per shot block (kFieldsPerShot fields)
    int tiles_x = 0, tiles_z = 0;
    int rec_x0 = 0, rec_z0 = 0, rec_tiles_x = 0, rec_tiles_z = 0;   // reconstruction tiles (TileGrid)
    float a[6] = {0, 0, 0, 0, 0, 0};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    std::string err;
    ouc_timing timing{};
    Ring ring{};
    std::vector<float> vp_host;  // padded Vp (for the mute's velocity)

    // device memory
    float* model = nullptr;      // 9 fields: vp2 vs2 ax az bx bz (moduli per unit density, or times rho), vp vs rho
    float* state = nullptr;      // batch shot blocks
    float *vp2 = nullptr, *vs2 = nullptr, *ax = nullptr, *az = nullptr;
    float *bx = nullptr, *bz = nullptr;   // buoyancy at the Ux / Uz positions (cfg.density)
    float *vpv = nullptr, *vsv = nullptr, *rhov = nullptr;   // Vp, Vs, rho (null without a rho model)
    // FWI gradient (cfg.gradient): per-shot accumulators [batch][3] and FP64 stacks
    float* grad = nullptr;
    double* d_gstack[3] = {nullptr, nullptr, nullptr};
    Side src{}, rcv{};
    Side src0{}, rcv0{};         // leapfrog buffer assignment the whole-shot loops start from
    // CUDA graphs of whole-shot time loops (cfg.use_graphs), keyed by loop
    // kind and flags; replayed for every later batch with the same key
    struct Graph {
        int key[6];
        cudaGraphExec_t exec;
        Side src_end;            // source side after the loop
        long long launches;      // kernels in the loop
    };
    std::vector<Graph> graphs;
    float* acc[3] = {nullptr, nullptr, nullptr};
    float* comp[3] = {nullptr, nullptr, nullptr};   // compensation terms of acc (compensated_image)
    float* gathers = nullptr;    // [batch][2][nt][X], time-major
    float* staging = nullptr;    // max(nt*X, 4*X*Z) floats for transposes / packing
    float* d_wavelet = nullptr;
    float* d_img = nullptr;      // [batch][2][nx][nz]
    double* d_stack[3] = {nullptr, nullptr, nullptr};
    void* strips = nullptr;      // [batch][nt][8][R] of the strip element type
    float* stage = nullptr;      // f16 strips: staging rings [batch][2][8][R]
    unsigned* amax = nullptr;    // f16 strips: per-slot field maxima [batch][nt][8]
    // snapshot form (cfg.snapshot_every = K >= 1)
    void* snaps = nullptr;       // [batch][nslots][2][nx][nz] of the strip element type
    unsigned* snap_amax = nullptr;   // f16: [batch][nslots][2]
    int nslots = 0;
    std::vector<int> snap_fwd;   // forward step -> snapshot slot of its new level, or -1
    std::vector<int> snap_bwd;   // backward step -> slot imaged there, or -1
    size_t strip_slot = 0;       // floats per slot
    ShotDesc* d_desc = nullptr;  // [batch]
    // learned corrector (learned.cu), allocated on first use
    float* l_in = nullptr;       // network input  [X][Z][OUC_CNN_IN]
    float* l_out = nullptr;      // network output [X][Z][OUC_CNN_OUT]
    float* l_truth = nullptr;    // restricted fine state, two levels [2][X][Z][4]
    float* l_scale = nullptr;    // [2] largest |U| and |U^n - U^(n-1)| of the state
    float* l_tmp = nullptr;      // [X][Z][OUC_CNN_OUT] smoothing scratch
    // survey (survey.cu): per-slot sub-grid models [batch][4 fields] (vp2 vs2 ax az)
    float* sv_model = nullptr;
    // first-order scheme (fo.cu): powf(Vp, 2), powf(Vs, 2) in the model layout, allocated on first use
    float* fo_sq = nullptr;
    size_t bytes = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t stream2 = nullptr;    // receiver steps of the overlapped backward loop
    cudaEvent_t evb[3] = {nullptr, nullptr, nullptr};   // its ordering events (no timing)

    // step-level interface: one shot (slot 0) advanced one launch per call
    enum { kIdle, kForward, kReceiver, kReconstruct, kFinalize } step_phase = kIdle;
    int step_t = 0;              // the time the next step call must name
    ouc_shot step_shot{};
    StepArgs step_fwd{}, step_rcv{}, step_rec{};

    float* field(float* base, size_t k) const { return base + k * fstride + (size_t)kGX * pitch + kZOFF; }
    float* gather(int b, int comp) const { return gathers + ((size_t)b * 2 + comp) * (size_t)nt * X; }
};

namespace ouc {
namespace host {

int fail(ouc_ctx* c, int code, const std::string& msg);
int cuda_fail(ouc_ctx* c, cudaError_t e, const char* what);
StepArgs base_args(const ouc_ctx* c);
void bind_side(StepArgs& a, const Side& s);
int check_shot(ouc_ctx* ctx, const ouc_shot* s);
// Upload the descriptors of n shots (interior coordinates in, padded stored).
int upload_desc(ouc_ctx* ctx, int n, const ouc_shot* shots, const float* d_wavelet);
// Zero one side's fields (0 source, 1 receiver) of n shots, optionally the imaging accumulators.
int zero_side(ouc_ctx* ctx, int n, int side, bool with_acc);
// One forward step of n shots at time t; swaps the leapfrog levels of `s`.
int fwd_step(ouc_ctx* ctx, StepArgs& a, Side& s, int n, int t);
int run_forward(ouc_ctx* ctx, int n, bool record, bool save, bool snaps = false);
int run_forward_loop(ouc_ctx* ctx, int n, bool record, bool save, bool snaps);
int gather_out(ouc_ctx* ctx, const float* src_tx, float* dst, bool host);
int gather_in(ouc_ctx* ctx, const float* src, float* dst_tx, bool host);
int ensure_strips(ouc_ctx* ctx);
int run_backward(ouc_ctx* ctx, int n, bool exact_strips, bool theta_src);
int run_backward_loop(ouc_ctx* ctx, int n, bool exact_strips, bool theta_src);
int run_backward_snap_loop(ouc_ctx* ctx, int n);
void damping(const std::vector<float>& vp, int X, int Z, int L, double R, std::vector<float>& ax,
             std::vector<float>& az);
float elapsed(cudaEvent_t a, cudaEvent_t b);
// Read and clear the device status word (after the stream's work): OUC_OK,
// OUC_ETIMEOUT or OUC_EUNSTABLE.
int check_status(ouc_ctx* ctx);

}  // namespace host
}  // namespace ouc
