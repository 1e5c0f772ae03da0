// rtm_engine.cu — host engine: sessions, device memory, batching of shots and the
// per-pass time loops (reference shot driver rtm_model.cu:117-569, re-designed so that a
// batch of shots shares every launch and all boundary strips stay in HBM).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "rtm_b200.h"
#include "rtm_internal.h"
#include "rtm_launch.h"
#include "rtm_types.h"

namespace rtm {

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(RTM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

static constexpr int kRing = 32;   // fp32 staging ring (steps) for reduced-precision strips

static size_t elem_size(int prec) { return prec == RTM_PREC_FP32 ? 4 : 2; }
static int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Device allocation arena: one cudaMalloc per session, 256-byte aligned sub-allocations.
// With guards on (RTM_B200_GUARDS=1, a checking mode) every sub-allocation is followed by at
// least kGuardBytes filled with kGuardByte on the session stream as it is taken, and
// check_guards() verifies them after setup and after every batch: a kernel that writes past
// the end of any buffer is reported with the buffer's label.
static constexpr size_t kGuardBytes = 256;
static constexpr int kGuardByte = 0xA5;
struct Arena {
    char *base = nullptr;
    size_t size = 0, used = 0;
    bool guard = false;
    cudaStream_t stream = nullptr;
    const char *label = "";
    struct Guard {
        size_t off, len;
        const char *label;
        int index;
    };
    std::vector<Guard> guards;
    int taken = 0;
    void *take(size_t n)
    {
        size_t off = (used + 255) & ~(size_t)255;
        const size_t tail = guard ? ((n + 255) & ~(size_t)255) - n + kGuardBytes : 0;
        if (off + n + tail > size) return nullptr;
        used = off + n + tail;
        if (guard) {
            guards.push_back({off + n, tail, label, taken});
            if (cudaMemsetAsync(base + off + n, kGuardByte, tail, stream) != cudaSuccess) return nullptr;
        }
        taken++;
        return base + off;
    }
};

struct ModelDev {       // one padded model pair on the device
    float *inv_rho = nullptr, *kappa = nullptr;
    float *vp2 = nullptr;  // v^2, kept only for the other imaging conditions
};

struct ShotState {
    int ishot = 0;
    rtm_geometry g{};
    int X = 0, Z = 0, pitch = 0, nxi = 0, nzi = 0, strip_len = 0;
    float vpmax = 0;
    int sbx0 = 0, sbz0 = 0, sbnx = 0, sbnz = 0;
    ModelDev mf, mb;
    float *pml = nullptr, *src = nullptr, *mute_row = nullptr;   // mute_row: v^2 row rz (+ v^2 at source)
    float *gather_raw = nullptr;      // mode 0: [nt][nrec] modelled gather, unmuted
    float *gather32 = nullptr;        // [nt][nrec] fp32 gather that is migrated (muted)
    void *gather_packed = nullptr;    // fp16/bf16 copy
    float *gather_scale = nullptr;
    bool gather_ready = false;
    std::vector<float> mute_row_host;
};

struct Slot {
    WaveDev a{}, b{};
    WaveDev a2{}, b2{};   // whole-step kernel: second buffers of p, vx, vz (sx, sz are a's and b's)
    void *strips = nullptr;
    float *strip_scale = nullptr, *strip_stage = nullptr;
    void *g1 = nullptr, *illum = nullptr;
    double *g1t = nullptr, *illt = nullptr;               // fp64 totals of the blocked accumulation
    void *gx[4] = {nullptr, nullptr, nullptr, nullptr};   // other imaging conditions (g2, g3, g3t, g4)
    float *ps_pre = nullptr, *p_pre = nullptr;           // pressures before the current backward step
};

struct KernelTiming {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    int used = 0;
};

}  // namespace rtm

struct rtm_session {
    rtm_survey s{};
    rtm_options o{};
    int dev = 0;
    cudaStream_t stream = nullptr;
    rtm::Arena arena;
    std::vector<rtm::ShotState> shots;
    std::vector<rtm::Slot> slots;
    int B = 0;                       // batch size (slots)
    int maxX = 0, maxPitch = 0, Z = 0;
    float *wavelet = nullptr, *coef = nullptr;
    float coef_host[100];
    void *img1 = nullptr, *img2s = nullptr, *img2m = nullptr, *illum = nullptr;
    void *ximg[7] = {};              // image3s, image4s, image5s, image3m, image4m, image5m, imagetrue
    ShotDev *d_shots = nullptr;
    TileRef *d_tiles = nullptr;      // tiles of the velocity kernels (whole padded grid)
    TileRef *d_tiles_p = nullptr;    // tiles of the pressure kernels (whole padded grid)
    TileRef *d_tiles_r = nullptr;    // velocity tiles of the reconstruction region (interior + strips)
    TileRef *d_tiles_pr = nullptr;   // pressure tiles of the reconstruction region
    // rows per tile (measured): 32 for the forward and receiver velocity kernels, 16 for the
    // velocity reconstruction and the pressure kernels (forward and receiver pressure share
    // one tile list; the pressure reconstruction has its own)
    int bz_vel = 32, bz_vel_recon = 16, bz_pres = 16, bz_pres_recon = 16;
    // kernel form per family (forward/receiver velocity, reconstruction velocity, forward/receiver
    // pressure, reconstruction pressure): four columns by U rows per thread (rtm_stencil_v.cu)
    // or one column per thread (rtm_stencil.cu); the results are the same bits.  Chosen by the
    // tuner with the tile heights; without it the measured defaults (one column per thread for
    // the full-grid kernels, four columns for the reconstruction), or all of one form with
    // RTM_B200_KERNELS=scalar|vector.
    bool vec[4] = {false, true, false, true};
    bool forms_fixed = false;
    bool tune = true;                // choose the tile heights per launch shape by timing them
    // whole-step kernel (rtm_step.cu): velocity and pressure of a step in one launch over
    // tz_step-row tiles, two buffers per field, four descriptor tables (which buffer is
    // current for each wavefield)
    bool fused = false;
    int tz_step = 32;
    // persistent passes (k_pass, RTM_B200_PERSIST=1): every step of a pass in one launch over a
    // device work queue with per-shot completion counters; one-column kernels at 32/16/16 rows
    bool persist = false;
    long long pass_wait_ns = 2000000000LL;   // bound on one wait (RTM_B200_PASS_WAIT_US)
    int *d_per_shot = nullptr;               // [6][B]: tiles per shot, source pass lists then backward lists
    unsigned *d_queue = nullptr, *d_done = nullptr;   // pass queue counter; [4][B] completion counters
    unsigned *d_trace = nullptr;             // the item each persistent block took last
    int trace_len = 0;
    void *d_fin = nullptr;
    void *d_tmaps = nullptr;         // B x RTM_TMAP_COUNT tensor maps (rebuilt for every batch)
    int *d_err = nullptr;            // kernel error flag (bounded waits that gave up)
    int *d_counts = nullptr;         // tile counts of the batch's four lists (fixed-grid launches)
    int max_tiles = 0;
    std::map<std::string, rtm::KernelTiming> timing;
    int launches = 0;
    int last_batch_n = 0;
    std::vector<int> last_batch_shots;
    rtm::InterpPlan interp;          // real-data path: workspace of the gather interpolation
    int *d_nonfinite = nullptr;      // lowest batch index of a shot whose image went non-finite
    unsigned *d_absmax = nullptr;    // progress snapshots: [2 passes][snaps][B] max |p| bits
    int nsnap = 0;                   // snapshots per pass (0: none)
    unsigned long long config_hash = 0;   // survey, image-relevant options, shots, models
    // use_graph: the time loop of each pass captured as one CUDA graph, instantiated once per
    // launch shape (batch size and tile counts) and replayed for every batch of that shape
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        int launches = 0;   // kernels per replay
    };
    std::map<std::vector<long>, GraphEntry> graphs;
    bool capturing = false;
};

namespace rtm {

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (no link to
// libcuda needed).
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Tensor map of one [Z][pitch] fp32 field for boxes of box_w x box_h elements.  Rows and
// columns outside the field read as zero (the stencil kernels rely on it at the grid edge).
static int encode_field_map(void *out, float *field, int pitch, int Z, int box_w, int box_h)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    if (!enc) return fail(RTM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    // TMA needs a 16-byte aligned base, a row stride that is a multiple of 16 bytes and a box
    // row of a multiple of 16 bytes; boxes are at most 256 elements per dimension
    if (((uintptr_t)field & 15) || (pitch * 4) % 16 || (box_w * 4) % 16 || box_w > 256 || box_h > 256)
        return fail(RTM_ERR_ARG, "tensor map: misaligned field or box");
    cuuint64_t dim[2] = {(cuuint64_t)pitch, (cuuint64_t)Z};
    cuuint64_t stride[1] = {(cuuint64_t)pitch * 4};
    cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = enc((CUtensorMap *)out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, field, dim, stride, box, estride,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(RTM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return RTM_OK;
}

// Read and clear the kernels' error flag (after the stream has been synchronised).
static int check_kernel_flag(rtm_session *ss)
{
    int e[8] = {};
    CK(cudaMemcpy(e, ss->d_err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e[0]) {
        CK(cudaMemset(ss->d_err, 0, sizeof(e)));
        if (e[0] == 2)
            return fail(RTM_ERR_CUDA, "a persistent pass gave up waiting for the work items of other blocks");
        char where[200] = "";
        if (e[1]) {
            unsigned item = 0;
            if (ss->persist && e[2] >= 0 && e[2] < ss->trace_len)
                cudaMemcpy(&item, ss->d_trace + e[2], sizeof(unsigned), cudaMemcpyDeviceToHost);
            std::snprintf(where, sizeof where, " (block %d, barrier at shared 0x%x, state 0x%08x%08x, persistent item %u)",
                          e[2], (unsigned)e[3], (unsigned)e[5], (unsigned)e[4], item);
        }
        return fail(RTM_ERR_CUDA, std::string("a stencil kernel gave up waiting for its tile (TMA copy did not complete)") +
                                      where);
    }
    return RTM_OK;
}

// FNV-1a, 64 bit.
static unsigned long long fnv1a(const void *data, size_t n, unsigned long long h = 1469598103934665603ULL)
{
    const unsigned char *p = (const unsigned char *)data;
    for (size_t i = 0; i < n; i++) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// After a batch: a shot whose image holds NaN or infinity stops the run with a status.
static int check_nonfinite(rtm_session *ss, int k0, int n)
{
    int bad = n;
    CK(cudaMemcpy(&bad, ss->d_nonfinite, sizeof(int), cudaMemcpyDeviceToHost));
    if (bad >= 0 && bad < n)
        return fail(RTM_ERR_NUMERIC, "shot " + std::to_string(ss->shots[k0 + bad].ishot) +
                                         ": the image holds NaN or infinite values (the wavefield diverged: time step "
                                         "above the stability limit, or invalid model values)");
    return RTM_OK;
}

// Guard bands of the checking mode: every byte must still hold kGuardByte.
static int check_guards(rtm_session *ss)
{
    if (!ss->arena.guard) return RTM_OK;
    CK(cudaStreamSynchronize(ss->stream));
    std::vector<unsigned char> h;
    for (const Arena::Guard &g : ss->arena.guards) {
        h.resize(g.len);
        CK(cudaMemcpy(h.data(), ss->arena.base + g.off, g.len, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < g.len; i++)
            if (h[i] != kGuardByte)
                return fail(RTM_ERR_CUDA, "device write " + std::to_string(i) + " bytes past the end of allocation #" +
                                              std::to_string(g.index) + " (" + g.label + ")");
    }
    return RTM_OK;
}

int session_guard_count(rtm_session *ss) { return ss ? (int)ss->arena.guards.size() : 0; }

static int check_survey(const rtm_survey &s)
{
    if (s.nx < 2 || s.nz < 2 || s.nt < 2) return fail(RTM_ERR_ARG, "nx, nz and nt must be >= 2");
    if (!(s.dx > 0) || !(s.dz > 0) || !(s.dt > 0)) return fail(RTM_ERR_ARG, "dx, dz and dt must be > 0");
    if (s.npml < RTM_RADIUS) return fail(RTM_ERR_ARG, "npml must be >= 10 (the stencil radius)");
    if (s.mode != 0 && s.mode != 1) return fail(RTM_ERR_ARG, "mode must be 0 or 1");
    if (s.receiver_depth < 0 || s.receiver_depth >= s.nz) return fail(RTM_ERR_ARG, "receiver_depth out of range");
    if (s.mute < 0 || s.mute > 2) return fail(RTM_ERR_ARG, "mute must be 0, 1 or 2");
    return RTM_OK;
}

// A caller-supplied shot geometry (the real-data path) must describe a window inside the
// model and nodes inside its padded grid.
static int check_geometry(const rtm_survey &s, const rtm_geometry &g, int ishot)
{
    const std::string who = "shot " + std::to_string(ishot) + ": ";
    if (g.nx1 < 0 || g.nx2 > s.nx - 1 || g.nx2 - g.nx1 + 1 != g.nxlength || g.nxlength < 2)
        return fail(RTM_ERR_ARG, who + "window outside the model");
    if (g.nxpad != g.nxlength + 2 * s.npml || g.nzpad != s.nz + 2 * s.npml)
        return fail(RTM_ERR_ARG, who + "padded grid does not match the window");
    if (g.nsx < 0 || g.nsx >= g.nxpad || g.nsz < 0 || g.nsz >= g.nzpad)
        return fail(RTM_ERR_ARG, who + "source outside its grid");
    if (g.nrec < 1 || g.rx0 < 0 || g.rx0 + g.nrec > g.nxpad || g.rz < 0 || g.rz >= g.nzpad)
        return fail(RTM_ERR_ARG, who + "receivers outside the grid");
    return RTM_OK;
}

// Padded model pair of one shot window: v^2 (squared in float, extractvel1) and rho,
// optionally PML-smoothed (medium_flag) and Gaussian-smoothed (ismth).
static void prep_model(const rtm_survey &s, const float *vp, const float *rho, int nx1, int nx2, bool smooth,
                       std::vector<float> &vp2, std::vector<float> &rp)
{
    const int nxl = nx2 - nx1 + 1, X = nxl + 2 * s.npml, Z = s.nz + 2 * s.npml;
    vp2.assign((size_t)X * Z, 0.0f);
    rp.assign((size_t)X * Z, 0.0f);
    extract_extend(vp, s.nx, s.nz, nx1, nx2, s.npml, true, vp2.data());
    extract_extend(rho, s.nx, s.nz, nx1, nx2, s.npml, false, rp.data());
    if (s.medium_flag) {
        pml_smooth(vp2.data(), X, Z, s.npml);
        pml_smooth(rp.data(), X, Z, s.npml);
    }
    if (smooth && s.ismth > 0) {
        gauss_smooth(vp2.data(), Z, X, s.ismth);
        gauss_smooth(rp.data(), Z, X, s.ismth);
    }
}

static int upload_model(rtm_session *ss, const std::vector<float> &vp2, const std::vector<float> &rho, int X, int Z,
                        int pitch, ModelDev &m)
{
    if (ss->o.extra_images) {   // v^2 for the Poynting and energy-norm imaging conditions
        std::vector<float> v((size_t)pitch * Z, 0.0f);
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) v[(size_t)z * pitch + x] = vp2[(size_t)z * X + x];
        m.vp2 = (float *)ss->arena.take(sizeof(float) * v.size());
        if (!m.vp2) return fail(RTM_ERR_NOMEM, "device arena exhausted (models)");
        CK(cudaMemcpyAsync(m.vp2, v.data(), sizeof(float) * v.size(), cudaMemcpyHostToDevice, ss->stream));
        CK(cudaStreamSynchronize(ss->stream));
    }
    std::vector<float> ir((size_t)pitch * Z, 0.0f), ka((size_t)pitch * Z, 0.0f);
    for (int z = 0; z < Z; z++)
        for (int x = 0; x < X; x++) {
            float r = rho[(size_t)z * X + x];
            ir[(size_t)z * pitch + x] = 1.0f / r;
            ka[(size_t)z * pitch + x] = r * vp2[(size_t)z * X + x];
        }
    m.inv_rho = (float *)ss->arena.take(sizeof(float) * ir.size());
    m.kappa = (float *)ss->arena.take(sizeof(float) * ka.size());
    if (!m.inv_rho || !m.kappa) return fail(RTM_ERR_NOMEM, "device arena exhausted (models)");
    CK(cudaMemcpyAsync(m.inv_rho, ir.data(), sizeof(float) * ir.size(), cudaMemcpyHostToDevice, ss->stream));
    CK(cudaMemcpyAsync(m.kappa, ka.data(), sizeof(float) * ka.size(), cudaMemcpyHostToDevice, ss->stream));
    CK(cudaStreamSynchronize(ss->stream));
    return RTM_OK;
}

// Bytes per cell of the per-shot accumulators g1 and illum that the imaging kernels update every
// step: fp32, fp64, a compensated fp32 pair, or the fp32 partial sums of the blocked form.
static int acc_bytes(const rtm_options &o)
{
    return o.accum_fp64 == RTM_ACC_FP64 || o.accum_fp64 == RTM_ACC_KAHAN ? 8 : 4;
}

static size_t slot_bytes(const rtm_survey &s, const rtm_options &o, int pitch, int Z, int strip_len, int nxi, int nzi,
                         bool fused)
{
    size_t field = (size_t)pitch * Z * sizeof(float) + 256;
    size_t b = (fused ? 16 : 10) * field;
    b += (size_t)s.nt * strip_len * elem_size(o.strip_precision) + 256;
    if (o.strip_precision != RTM_PREC_FP32) {
        b += (size_t)s.nt * 4 * sizeof(float) + 256;
        b += (size_t)kRing * strip_len * sizeof(float) + 256;
    }
    b += 2 * ((size_t)pitch * Z * acc_bytes(o) + 256);   // g1, illum on the padded grid
    if (o.accum_fp64 == RTM_ACC_FP64_BLOCKED) b += 2 * ((size_t)pitch * Z * 8 + 256);   // their fp64 totals
    if (o.extra_images) b += 4 * ((size_t)pitch * Z * (o.accum_fp64 ? 8 : 4) + 256) + 2 * field;
    (void)nxi;
    (void)nzi;
    return b;
}

static int open_session(rtm_session *ss, const float *vp, const float *rho, const float *vp_mig,
                        const float *rho_mig, const float *diffcoef, const int *shot_ids, int nshots,
                        const rtm_geometry *geoms = nullptr)
{
    const rtm_survey &s = ss->s;
    const rtm_options &o = ss->o;
    int rc = check_survey(s);
    if (rc) return rc;
    if (nshots < 1) return fail(RTM_ERR_ARG, "no shots");
    CK(cudaSetDevice(o.device));
    ss->dev = o.device;
    CK(cudaStreamCreateWithFlags(&ss->stream, cudaStreamNonBlocking));

    // geometry and sizes of every shot
    ss->shots.resize(nshots);
    size_t shot_bytes_total = 0;
    ss->Z = s.nz + 2 * s.npml;
    for (int k = 0; k < nshots; k++) {
        ShotState &sh = ss->shots[k];
        sh.ishot = shot_ids[k];
        if (geoms) {
            sh.g = geoms[k];
            rc = check_geometry(s, sh.g, sh.ishot);
        } else {
            rc = shot_geometry(s, sh.ishot, sh.g);
        }
        if (rc) return rc;
        sh.X = sh.g.nxpad;
        sh.Z = sh.g.nzpad;
        sh.pitch = round_up(sh.X, 32);
        sh.nxi = sh.g.nxlength;
        sh.nzi = s.nz;
        sh.strip_len = 2 * RTM_RADIUS * (sh.nzi + sh.nxi) * 2;
        ss->maxX = std::max(ss->maxX, sh.X);
        ss->maxPitch = std::max(ss->maxPitch, sh.pitch);
        size_t gb = (size_t)s.nt * sh.g.nrec;
        shot_bytes_total += (s.mode == 0 ? 2 : 1) * (gb * 4 + 256);
        if (o.gather_precision != RTM_PREC_FP32) shot_bytes_total += gb * 2 + (size_t)s.nt * 4 + 512;
        shot_bytes_total += (size_t)pml_offsets(sh.X, sh.Z).total * 4 + 256 + (size_t)(sh.X + 1) * 4 + 256;
    }
    // source stamp boxes: cells where amp*expf(-alp^2*dist) can be non-zero
    for (ShotState &sh : ss->shots) {
        int hx = sh.X, hz = sh.Z;
        if (s.alp != 0.0f) {
            double r = std::sqrt(104.0 / ((double)s.alp * s.alp));
            hx = (int)(r / s.dx) + 2;
            hz = (int)(r / s.dz) + 2;
        }
        sh.sbx0 = std::max(0, sh.g.nsx - hx);
        sh.sbz0 = std::max(0, sh.g.nsz - hz);
        int x1 = std::min(sh.X - 1, sh.g.nsx + hx), z1 = std::min(sh.Z - 1, sh.g.nsz + hz);
        sh.sbnx = x1 - sh.sbx0 + 1;
        sh.sbnz = z1 - sh.sbz0 + 1;
        shot_bytes_total += (size_t)sh.sbnx * sh.sbnz * 4 + 256;
    }
    // models: one padded pair per distinct window (layout 2 shares one for every shot)
    std::map<std::pair<int, int>, int> windows;
    for (ShotState &sh : ss->shots) windows[{sh.g.nx1, sh.g.nx2}] = 0;
    const bool sep_b = (vp_mig != nullptr) || (s.ismth > 0);
    size_t model_bytes = 0;
    for (auto &w : windows) {
        int X = w.first.second - w.first.first + 1 + 2 * s.npml;
        model_bytes += ((sep_b ? 4 : 2) + (o.extra_images ? (sep_b ? 2 : 1) : 0)) *
                       ((size_t)round_up(X, 32) * ss->Z * 4 + 256);
    }
    // device memory plan
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const ShotState &big = *std::max_element(ss->shots.begin(), ss->shots.end(),
                                             [](const ShotState &a, const ShotState &b) { return a.X < b.X; });
    {
        // RTM_B200_FUSED=1: the whole-step kernel; RTM_B200_TZ_STEP: its rows per tile (16, 32)
        const char *e = std::getenv("RTM_B200_FUSED");
        if (e && *e) ss->fused = std::atoi(e) != 0;
        if ((e = std::getenv("RTM_B200_TZ_STEP")) && *e) {
            ss->tz_step = std::atoi(e);
            ss->tune = false;
        }
        if (ss->tz_step != 16 && ss->tz_step != 32) return fail(RTM_ERR_ARG, "RTM_B200_TZ_STEP must be 16 or 32");
        if ((e = std::getenv("RTM_B200_PERSIST")) && *e) ss->persist = std::atoi(e) != 0 && !ss->fused;
        if ((e = std::getenv("RTM_B200_PASS_WAIT_US")) && *e) ss->pass_wait_ns = std::atoll(e) * 1000LL;
    }
    size_t per_slot = slot_bytes(s, o, big.pitch, big.Z, big.strip_len, big.nxi, big.nzi, ss->fused);
    size_t fixed = model_bytes + shot_bytes_total + (o.extra_images ? 11 : 4) * ((size_t)s.nx * s.nz * 8 + 256) + (size_t)s.nt * 4 + 4096 +
                   (size_t)(64 << 20);
    size_t budget = (size_t)(free_b * 0.92);
    if (fixed + per_slot > budget) return fail(RTM_ERR_NOMEM, "survey does not fit in device memory");
    int B = (int)std::min<size_t>((size_t)nshots, (budget - fixed) / per_slot);
    if (o.batch > 0) B = std::min(B, o.batch);
    {
        const char *e = std::getenv("RTM_B200_BZ_VEL");
        if (e && *e) ss->bz_vel = std::atoi(e);
        e = std::getenv("RTM_B200_BZ_VEL_RECON");
        if (e && *e) ss->bz_vel_recon = std::atoi(e);
        e = std::getenv("RTM_B200_BZ_PRES");
        if (e && *e) ss->bz_pres = ss->bz_pres_recon = std::atoi(e);
        e = std::getenv("RTM_B200_BZ_PRES_RECON");
        if (e && *e) ss->bz_pres_recon = std::atoi(e);
        // tile heights set by hand turn the tuner off; so does RTM_B200_TUNE=0
        for (const char *v : {"RTM_B200_BZ_VEL", "RTM_B200_BZ_VEL_RECON", "RTM_B200_BZ_PRES", "RTM_B200_BZ_PRES_RECON"})
            if ((e = std::getenv(v)) && *e) ss->tune = false;
        if ((e = std::getenv("RTM_B200_TUNE")) && *e && std::atoi(e) == 0) ss->tune = false;
        e = std::getenv("RTM_B200_KERNELS");
        if (e && *e) {
            if (std::strcmp(e, "scalar") && std::strcmp(e, "vector"))
                return fail(RTM_ERR_ARG, "RTM_B200_KERNELS must be scalar or vector");
            for (bool &v : ss->vec) v = !std::strcmp(e, "vector");
            ss->forms_fixed = true;
        }
        if (ss->persist) {   // the persistent passes run the one-column kernels at the default heights
            ss->tune = false;
            ss->bz_vel = 32;
            ss->bz_vel_recon = 16;
            ss->bz_pres = ss->bz_pres_recon = 16;
            for (bool &v : ss->vec) v = false;
        }
        if (o.extra_images < 0 || o.extra_images > 2) return fail(RTM_ERR_ARG, "extra_images must be 0, 1 or 2");
        if (o.accum_fp64 < 0 || o.accum_fp64 > 3) return fail(RTM_ERR_ARG, "accum_fp64 must be 0, 1, 2 or 3");
        for (int bz : {ss->bz_vel, ss->bz_vel_recon, ss->bz_pres, ss->bz_pres_recon})
            if (bz != 8 && bz != 16 && bz != 32 && bz != 64) return fail(RTM_ERR_ARG, "tile heights must be 8, 16, 32 or 64");
    }
    B = std::max(B, 1);
    ss->B = B;
    size_t arena_bytes = fixed + (size_t)B * per_slot;
    {
        const char *g = std::getenv("RTM_B200_GUARDS");
        ss->arena.guard = g && std::atoi(g) != 0;
    }
    if (ss->arena.guard)   // an upper bound of the sub-allocations, each with its guard
        arena_bytes += (size_t)(16 * nshots + 8 * (int)windows.size() + 32 * B + 64) * (kGuardBytes + 256);
    char *base = nullptr;
    CK(cudaMalloc((void **)&base, arena_bytes));
    ss->arena.base = base;
    ss->arena.size = arena_bytes;
    ss->arena.stream = ss->stream;
    ss->arena.label = "wavelet and coefficients";

    // wavelet and coefficient table
    ss->wavelet = (float *)ss->arena.take((size_t)s.nt * 4);
    ss->coef = (float *)ss->arena.take(100 * 4);
    launch_ricker(ss->wavelet, s.fdom, s.dt, s.nt, ss->stream);
    ss->launches++;
    float ctab[100];
    if (diffcoef) std::memcpy(ctab, diffcoef, sizeof(ctab));
    else coef_table(ctab);
    std::memcpy(ss->coef_host, ctab, sizeof(ctab));
    CK(cudaMemcpyAsync(ss->coef, ctab, sizeof(ctab), cudaMemcpyHostToDevice, ss->stream));
    CK(cudaStreamSynchronize(ss->stream));
    // stacked images
    ss->arena.label = "stacked images";
    const size_t isz = (size_t)s.nx * s.nz * (o.accum_fp64 ? 8 : 4);
    ss->img1 = ss->arena.take(isz);
    ss->img2s = ss->arena.take(isz);
    ss->img2m = ss->arena.take(isz);
    ss->illum = ss->arena.take(isz);
    CK(cudaMemsetAsync(ss->img1, 0, isz, ss->stream));
    CK(cudaMemsetAsync(ss->img2s, 0, isz, ss->stream));
    CK(cudaMemsetAsync(ss->img2m, 0, isz, ss->stream));
    CK(cudaMemsetAsync(ss->illum, 0, isz, ss->stream));
    if (o.extra_images)
        for (void *&im : ss->ximg) {
            if (!(im = ss->arena.take(isz))) return fail(RTM_ERR_NOMEM, "device arena exhausted (images)");
            CK(cudaMemsetAsync(im, 0, isz, ss->stream));
        }

    // models
    ss->arena.label = "models";
    std::map<std::pair<int, int>, std::pair<ModelDev, ModelDev>> mcache;
    std::map<std::pair<int, int>, std::pair<float, std::vector<float>>> vp2cache;
    std::map<std::pair<int, int>, std::vector<float>> vb2cache;   // mute 2: v^2 of the migration model
    for (auto &w : windows) {
        std::vector<float> vp2, rp;
        const int nx1 = w.first.first, nx2 = w.first.second;
        const int X = nx2 - nx1 + 1 + 2 * s.npml, pitch = round_up(X, 32);
        prep_model(s, vp, rho, nx1, nx2, false, vp2, rp);
        float m = vp2[0];
        for (float v : vp2) m = v > m ? v : m;
        ModelDev mf, mb;
        rc = upload_model(ss, vp2, rp, X, ss->Z, pitch, mf);
        if (rc) return rc;
        mb = mf;
        if (sep_b) {
            std::vector<float> vb2, rb;
            prep_model(s, vp_mig ? vp_mig : vp, rho_mig ? rho_mig : (vp_mig ? rho : rho), nx1, nx2, true, vb2, rb);
            rc = upload_model(ss, vb2, rb, X, ss->Z, pitch, mb);
            if (rc) return rc;
            if (s.mute == 2) vb2cache[w.first] = std::move(vb2);
        }
        mcache[w.first] = {mf, mb};
        vp2cache[w.first] = {sqrtf(m), std::move(vp2)};
    }
    // per-shot device state
    ss->arena.label = "per-shot state (PML, source, mute row, gathers)";
    for (ShotState &sh : ss->shots) {
        auto key = std::make_pair(sh.g.nx1, sh.g.nx2);
        sh.mf = mcache[key].first;
        sh.mb = mcache[key].second;
        sh.vpmax = vp2cache[key].first;
        // the direct-wave mute reads v^2 of the modelling model (rtm_model.cu mutes before
        // smoothing) or, with mute 2, of the migration model (rtm_real.cu:397-403 mutes after)
        const std::vector<float> &v2 = (s.mute == 2 && vb2cache.count(key)) ? vb2cache[key] : vp2cache[key].second;
        PmlOffsets po = pml_offsets(sh.X, sh.Z);
        sh.pml = (float *)ss->arena.take((size_t)po.total * 4);
        sh.src = (float *)ss->arena.take((size_t)sh.sbnx * sh.sbnz * 4);
        sh.mute_row = (float *)ss->arena.take((size_t)(sh.X + 1) * 4);
        size_t gb = (size_t)s.nt * sh.g.nrec;
        sh.gather32 = (float *)ss->arena.take(gb * 4);
        if (s.mode == 0) {
            sh.gather_raw = (float *)ss->arena.take(gb * 4);
            if (!sh.gather_raw) return fail(RTM_ERR_NOMEM, "device arena exhausted (gathers)");
            CK(cudaMemsetAsync(sh.gather_raw, 0, gb * 4, ss->stream));
        }
        if (o.gather_precision != RTM_PREC_FP32) {
            sh.gather_packed = ss->arena.take(gb * 2);
            sh.gather_scale = (float *)ss->arena.take((size_t)s.nt * 4);
        }
        if (!sh.pml || !sh.src || !sh.mute_row || !sh.gather32 ||
            (o.gather_precision != RTM_PREC_FP32 && (!sh.gather_packed || !sh.gather_scale)))
            return fail(RTM_ERR_NOMEM, "device arena exhausted (shots)");
        launch_setup_pml(sh.pml, sh.X, sh.Z, s.npml, s.dx, s.dz, s.dt, sh.vpmax, ss->stream);
        launch_setup_source(sh.src, sh.sbx0, sh.sbz0, sh.sbnx, sh.sbnz, sh.g.nsx, sh.g.nsz, s.amp, s.alp,
                            s.dx * s.dx, s.dz * s.dz, s.dt, ss->stream);
        ss->launches += 2;
        sh.mute_row_host.assign(sh.X + 1, 0.0f);
        for (int x = 0; x < sh.X; x++) sh.mute_row_host[x] = v2[(size_t)sh.g.rz * sh.X + x];
        sh.mute_row_host[sh.X] = v2[(size_t)sh.g.nsz * sh.X + sh.g.nsx];
        CK(cudaMemcpyAsync(sh.mute_row, sh.mute_row_host.data(), sizeof(float) * (sh.X + 1), cudaMemcpyHostToDevice,
                           ss->stream));
        CK(cudaMemsetAsync(sh.gather32, 0, gb * 4, ss->stream));
        CK(cudaStreamSynchronize(ss->stream));
    }
    // batch slots
    ss->arena.label = "batch slots (wavefields, strips, accumulators)";
    ss->slots.resize(B);
    for (Slot &sl : ss->slots) {
        const size_t fb = (size_t)big.pitch * big.Z * 4;
        float **f[16] = {&sl.a.p,  &sl.a.vx,  &sl.a.vz,  &sl.a.sx, &sl.a.sz, &sl.b.p, &sl.b.vx, &sl.b.vz,
                         &sl.b.sx, &sl.b.sz,  &sl.a2.p,  &sl.a2.vx, &sl.a2.vz, &sl.b2.p, &sl.b2.vx, &sl.b2.vz};
        for (int i = 0; i < (ss->fused ? 16 : 10); i++) {
            *f[i] = (float *)ss->arena.take(fb);
            if (!*f[i]) return fail(RTM_ERR_NOMEM, "device arena exhausted (fields)");
        }
        sl.a2.sx = sl.a.sx;
        sl.a2.sz = sl.a.sz;
        sl.b2.sx = sl.b.sx;
        sl.b2.sz = sl.b.sz;
        sl.strips = ss->arena.take((size_t)s.nt * big.strip_len * elem_size(o.strip_precision));
        if (o.strip_precision != RTM_PREC_FP32) {
            sl.strip_scale = (float *)ss->arena.take((size_t)s.nt * 4 * 4);
            sl.strip_stage = (float *)ss->arena.take((size_t)kRing * big.strip_len * 4);
        }
        const size_t cells = (size_t)big.pitch * big.Z, ib = cells * (o.accum_fp64 ? 8 : 4);
        sl.g1 = ss->arena.take(cells * acc_bytes(o));
        sl.illum = ss->arena.take(cells * acc_bytes(o));
        if (!sl.strips || !sl.g1 || !sl.illum) return fail(RTM_ERR_NOMEM, "device arena exhausted (slots)");
        if (o.accum_fp64 == RTM_ACC_FP64_BLOCKED) {
            sl.g1t = (double *)ss->arena.take(cells * 8);
            sl.illt = (double *)ss->arena.take(cells * 8);
            if (!sl.g1t || !sl.illt) return fail(RTM_ERR_NOMEM, "device arena exhausted (slots)");
        }
        if (o.extra_images) {
            for (void *&g : sl.gx)
                if (!(g = ss->arena.take(ib))) return fail(RTM_ERR_NOMEM, "device arena exhausted (slots)");
            sl.ps_pre = (float *)ss->arena.take((size_t)big.pitch * big.Z * 4);
            sl.p_pre = (float *)ss->arena.take((size_t)big.pitch * big.Z * 4);
            if (!sl.ps_pre || !sl.p_pre) return fail(RTM_ERR_NOMEM, "device arena exhausted (slots)");
        }
    }
    // descriptor and tile tables, tensor maps, kernel error flag
    ss->arena.label = "tables and flags";
    ss->d_shots = (ShotDev *)ss->arena.take(sizeof(ShotDev) * B * (ss->fused ? 4 : 1));
    ss->d_tmaps = ss->arena.take((size_t)B * RTM_TMAP_COUNT * RTM_TMAP_BYTES);
    ss->d_err = (int *)ss->arena.take(8 * sizeof(int));
    ss->d_nonfinite = (int *)ss->arena.take(sizeof(int));
    if (!ss->d_tmaps || !ss->d_err || !ss->d_nonfinite) return fail(RTM_ERR_NOMEM, "device arena exhausted (tables)");
    if (o.verbose && o.tsnap > 0.0f) {
        const int ntsnap = (int)(o.tsnap / s.dt);   // rtm_model.cu:21
        if (ntsnap >= 1) {
            ss->nsnap = (s.nt + ntsnap - 1) / ntsnap;
            ss->d_absmax = (unsigned *)ss->arena.take(sizeof(unsigned) * 2 * ss->nsnap * B);
            if (!ss->d_absmax) return fail(RTM_ERR_NOMEM, "device arena exhausted (snapshots)");
        }
    }
    CK(cudaMemsetAsync(ss->d_err, 0, 8 * sizeof(int), ss->stream));
    // tile tables sized for the shortest tile height the tuner or the environment may choose
    const int bz_min = 8;
    int tiles_per_shot = ((big.X + RTM_BX - 1) / RTM_BX + 1) * ((big.Z + bz_min - 1) / bz_min + 1);
    ss->max_tiles = tiles_per_shot * B;
    ss->d_tiles = (TileRef *)ss->arena.take(sizeof(TileRef) * ss->max_tiles);
    ss->d_tiles_p = (TileRef *)ss->arena.take(sizeof(TileRef) * ss->max_tiles);
    ss->d_tiles_r = (TileRef *)ss->arena.take(sizeof(TileRef) * ss->max_tiles);
    ss->d_tiles_pr = (TileRef *)ss->arena.take(sizeof(TileRef) * ss->max_tiles);
    ss->d_fin = ss->arena.take(finalize_shot_size() * B);
    ss->d_counts = (int *)ss->arena.take(4 * sizeof(int));
    ss->d_per_shot = (int *)ss->arena.take(6 * sizeof(int) * B);
    ss->d_queue = (unsigned *)ss->arena.take(2 * sizeof(unsigned));
    ss->d_done = (unsigned *)ss->arena.take(4 * sizeof(unsigned) * B);
    ss->trace_len = 148 * 16;
    ss->d_trace = (unsigned *)ss->arena.take(sizeof(unsigned) * ss->trace_len);
    if (!ss->d_counts || !ss->d_per_shot || !ss->d_queue || !ss->d_done)
        return fail(RTM_ERR_NOMEM, "device arena exhausted (tables)");
    if (!ss->d_shots || !ss->d_tiles || !ss->d_tiles_p || !ss->d_tiles_r || !ss->d_tiles_pr || !ss->d_fin)
        return fail(RTM_ERR_NOMEM, "device arena exhausted (tables)");
    CK(cudaStreamSynchronize(ss->stream));
    // what a checkpoint must agree on: the survey, the options that change the images, the
    // shots and their geometry, the models and the coefficients
    {
        const size_t nm = (size_t)s.nx * s.nz;
        unsigned long long h = fnv1a(&s, sizeof(s));
        const int oi[4] = {o.strip_precision, o.gather_precision, o.accum_fp64, o.extra_images};
        h = fnv1a(oi, sizeof(oi), h);
        for (const ShotState &sh : ss->shots) {
            h = fnv1a(&sh.ishot, sizeof(int), h);
            h = fnv1a(&sh.g, sizeof(sh.g), h);
        }
        h = fnv1a(vp, nm * sizeof(float), h);
        h = fnv1a(rho, nm * sizeof(float), h);
        if (vp_mig) h = fnv1a(vp_mig, nm * sizeof(float), h);
        if (rho_mig) h = fnv1a(rho_mig, nm * sizeof(float), h);
        h = fnv1a(ss->coef_host, sizeof(ss->coef_host), h);
        ss->config_hash = h;
    }
    return check_guards(ss);
}

// Mute the fp32 gather of shot k in place (reference kernel.cu:96-173) and pack it to the
// storage precision.
static int finish_gather(rtm_session *ss, ShotState &sh)
{
    const rtm_survey &s = ss->s;
    if (s.mode == 0)
        CK(cudaMemcpyAsync(sh.gather32, sh.gather_raw, sizeof(float) * (size_t)s.nt * sh.g.nrec,
                           cudaMemcpyDeviceToDevice, ss->stream));
    if (s.mute) {
        int nw = (int)(s.direct / (s.fdom * s.dt));   // rtm_model.cu:22-23
        int tlength = (int)(s.direct0 / s.dt);
        float rdt = (float)(1.0 / s.dt);
        launch_mute(sh.gather32, sh.mute_row, sh.X, sh.g.nsx, sh.g.nsz, s.nt, sh.g.rz, sh.g.rx0, sh.g.nrec, nw,
                    tlength, s.dx * s.dx, s.dz * s.dz, rdt, ss->stream);
        ss->launches++;
    }
    if (ss->o.gather_precision != RTM_PREC_FP32) {
        launch_gather_pack(sh.gather32, sh.gather_packed, sh.gather_scale, s.nt, sh.g.nrec, ss->o.gather_precision,
                           ss->stream);
        ss->launches++;
    }
    sh.gather_ready = true;
    CK(cudaGetLastError());
    return RTM_OK;
}

static void timing_begin(rtm_session *ss, const char *name, int it, cudaEvent_t *ev_end)
{
    *ev_end = nullptr;
    if (it % 64 != 7 || ss->capturing) return;   // events in a captured graph do not time
    KernelTiming &t = ss->timing[name];
    if (t.used == (int)t.ev.size()) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        t.ev.push_back({a, b});
    }
    cudaEventRecord(t.ev[t.used].first, ss->stream);
    *ev_end = t.ev[t.used].second;
    t.used++;
}
static void timing_end(rtm_session *ss, cudaEvent_t ev)
{
    if (ev) cudaEventRecord(ev, ss->stream);
}

// Batch state shared by the phases of one batch.
struct BatchRun {
    int k0 = 0, n = 0, ntiles = 0, ntiles_p = 0, ntiles_r = 0, ntiles_pr = 0, maxrec = 0, max_strip_len = 0;
    std::vector<ShotDev> hd;
    StepArgs a{};
    // whole-step kernel: which buffer holds the current source (pa) and receiver (pb) fields
    int pa = 0, pb = 0;
    // grid of the launches over each tile list: its tile count, or with use_graph that count
    // rounded up to four significant bits, so that one captured graph serves batches whose
    // windows differ a little; likewise the strip kernels' and the other imaging conditions'
    // extents
    int grid[4] = {0, 0, 0, 0};
    int strip_grid = 0, ex_nxi = 0, ex_nzi = 0;
};

// Launch arguments of a stencil launch over tile list L: the grid, and in fixed-grid mode the
// device tile counts that the blocks past the batch's tiles check.
static int list_grid(rtm_session *ss, BatchRun &br, StepArgs &a, int L)
{
    a.counts = ss->o.use_graph == 2 ? ss->d_counts : nullptr;
    a.list = L;
    return br.grid[L];
}

// Descriptor tables of a batch.  One table (hd as built) for the split kernels; with the
// whole-step kernel four, one per (pa, pb): in table 2 pa + pb, `a` is the source wavefield's
// buffer pa and `an` the other one, likewise b / bn with pb, so every kernel reads the current
// fields through `a` and `b` whatever the step.
static ShotDev *table(rtm_session *ss, const BatchRun &br) { return ss->d_shots + (size_t)(2 * br.pa + br.pb) * ss->B; }

static int upload_tables(rtm_session *ss, const BatchRun &br)
{
    const int n = br.n;
    if (!ss->fused) {
        CK(cudaMemcpyAsync(ss->d_shots, br.hd.data(), sizeof(ShotDev) * n, cudaMemcpyHostToDevice, ss->stream));
        return RTM_OK;
    }
    std::vector<ShotDev> t(4 * (size_t)ss->B);
    for (int pa = 0; pa < 2; pa++)
        for (int pb = 0; pb < 2; pb++)
            for (int j = 0; j < n; j++) {
                ShotDev d = br.hd[j];
                const WaveDev A0 = br.hd[j].a, A1 = br.hd[j].an, B0 = br.hd[j].b, B1 = br.hd[j].bn;
                d.a = pa ? A1 : A0;
                d.an = pa ? A0 : A1;
                d.b = pb ? B1 : B0;
                d.bn = pb ? B0 : B1;
                d.par_a = pa;
                d.par_b = pb;
                t[(size_t)(2 * pa + pb) * ss->B + j] = d;
            }
    CK(cudaMemcpyAsync(ss->d_shots, t.data(), sizeof(ShotDev) * t.size(), cudaMemcpyHostToDevice, ss->stream));
    // the host copy must live until the copy has read it
    CK(cudaStreamSynchronize(ss->stream));
    return RTM_OK;
}

// The tiles of one shot (batch slot j) in the four lists of a batch: 0 full-grid velocity
// (whole-step kernel: full-grid interior tiles), 1 full-grid pressure (whole-step: the other
// full-grid tiles), 2 reconstruction velocity (whole-step: interior tiles of the
// reconstruction region), 3 reconstruction pressure (whole-step: the other tiles there).
static void shot_tiles(const rtm_session *ss, const ShotState &sh, int j, bool fast, std::vector<TileRef> *const L[4])
{
    const rtm_survey &s = ss->s;
    std::vector<TileRef> &tiles = *L[0], &tiles_p = *L[1], &tiles_r = *L[2], &tiles_pr = *L[3];
    // whole-grid tiles, and the reconstruction's tiles: it writes only the interior and the
    // ten-cell strips around it, x in [npml-10, X-npml+10), z in [npml-10, Z-npml+10).  The
    // reconstruction's tile columns start on a 32-column (128-byte) boundary, so that every
    // warp's row access covers whole 128-byte lines, unless the 4-column boundary nearest
    // below the region needs one tile column fewer (the kernels skip the columns outside the
    // region)
    const int xr1 = sh.X - s.npml + RTM_RADIUS, xlo = s.npml - RTM_RADIUS;
    const int xr0 = (xr1 - (xlo & ~31) + RTM_BX - 1) / RTM_BX <= (xr1 - (xlo & ~3) + RTM_BX - 1) / RTM_BX
                        ? xlo & ~31 : xlo & ~3;
    const int zr0 = s.npml - RTM_RADIUS, zr1 = sh.Z - s.npml + RTM_RADIUS;
    // velocity tiles: interior when every column lies in [npml, X-npml-1) and every row in
    // [npml, Z-npml-1), where the velocity damping is 1 and no strip lies
    auto add_tiles = [&](std::vector<TileRef> &v, int bz, int xa, int xb, int za, int zb) {
        for (int z0 = za; z0 < zb; z0 += bz)
            for (int x0 = xa; x0 < xb; x0 += RTM_BX) {
                const bool inside = x0 >= s.npml && x0 + RTM_BX <= sh.X - s.npml - 1 && z0 >= s.npml &&
                                    z0 + bz <= sh.Z - s.npml - 1;
                v.push_back({j, x0, z0, (fast && inside) ? 1 : 0});
            }
    };
    if (ss->fused) {
        // whole-step tiles of tz_step rows, interior ones (cells and velocity halo in the
        // interior, full orders, no source or receiver) in their own lists: full grid
        // (fast: tiles, others: tiles_p) and reconstruction region (tiles_r, tiles_pr)
        const int tz = ss->tz_step, np = std::max(s.npml, RTM_RADIUS);
        auto fast_tile = [&](int x0, int z0, bool recon) {
            const bool vel_in = x0 - 12 >= np && x0 + RTM_BX + 12 <= sh.X - np - 1 && z0 - 10 >= np &&
                                z0 + tz + 10 <= sh.Z - np - 1;
            const bool src = x0 < sh.sbx0 + sh.sbnx && sh.sbx0 < x0 + RTM_BX && z0 < sh.sbz0 + sh.sbnz &&
                             sh.sbz0 < z0 + tz;
            const bool rec = !recon && sh.g.rz >= z0 && sh.g.rz < z0 + tz && x0 < sh.g.rx0 + sh.g.nrec &&
                             sh.g.rx0 < x0 + RTM_BX;
            return fast && vel_in && !src && !rec;
        };
        for (int z0 = 0; z0 < sh.Z; z0 += tz)
            for (int x0 = 0; x0 < sh.X; x0 += RTM_BX)
                (fast_tile(x0, z0, false) ? tiles : tiles_p).push_back({j, x0, z0, 1});
        for (int z0 = zr0; z0 < zr1; z0 += tz)
            for (int x0 = xr0; x0 < xr1; x0 += RTM_BX)
                (fast_tile(x0, z0, true) ? tiles_r : tiles_pr).push_back({j, x0, z0, 1});
    }
    if (!ss->fused) add_tiles(tiles, ss->bz_vel, 0, sh.X, 0, sh.Z);
    // pressure tiles: interior tiles (no PML, source or receiver cell) go to their own list
    for (int z0 = 0; z0 < (ss->fused ? 0 : sh.Z); z0 += ss->bz_pres)
        for (int x0 = 0; x0 < sh.X; x0 += RTM_BX) {
            const int x1 = x0 + RTM_BX, z1 = z0 + ss->bz_pres;
            const bool inside = x0 >= s.npml && x1 <= sh.X - s.npml && z0 >= s.npml && z1 <= sh.Z - s.npml;
            const bool src = x0 < sh.sbx0 + sh.sbnx && sh.sbx0 < x1 && z0 < sh.sbz0 + sh.sbnz && sh.sbz0 < z1;
            const bool rec = sh.g.rz >= z0 && sh.g.rz < z1 && x0 < sh.g.rx0 + sh.g.nrec && sh.g.rx0 < x1;
            tiles_p.push_back({j, x0, z0, (fast && inside && !src && !rec) ? 1 : 0});
        }
    if (!ss->fused) add_tiles(tiles_r, ss->bz_vel_recon, xr0, xr1, zr0, zr1);
    // reconstruction pressure tiles: interior when inside the pressure interior with no
    // source cell
    for (int z0 = zr0; z0 < (ss->fused ? zr0 : zr1); z0 += ss->bz_pres_recon)
        for (int x0 = xr0; x0 < xr1; x0 += RTM_BX) {
            const int x1 = x0 + RTM_BX, z1 = z0 + ss->bz_pres_recon;
            const bool inside = x0 >= s.npml && x1 <= sh.X - s.npml && z0 >= s.npml && z1 <= sh.Z - s.npml;
            const bool src = x0 < sh.sbx0 + sh.sbnx && sh.sbx0 < x1 && z0 < sh.sbz0 + sh.sbnz && sh.sbz0 < z1;
            tiles_pr.push_back({j, x0, z0, (fast && inside && !src) ? 1 : 0});
        }
}

// Bind shots [k0, k0+n) to slots 0..n-1, zero their wavefields and accumulators, upload
// the descriptor and (shot, tile) tables.
static int batch_setup(rtm_session *ss, int k0, int n, BatchRun &br)
{
    const rtm_survey &s = ss->s;
    const rtm_options &o = ss->o;
    cudaStream_t st = ss->stream;
    br.k0 = k0;
    br.n = n;
    br.hd.assign(n, ShotDev{});
    std::vector<TileRef> tiles, tiles_p, tiles_r, tiles_pr;
    const char *fast_env = std::getenv("RTM_B200_FAST_TILES");   // 0: every tile on the general form
    const bool fast = !(fast_env && *fast_env && std::atoi(fast_env) == 0);
    std::vector<unsigned char> maps((size_t)n * RTM_TMAP_COUNT * RTM_TMAP_BYTES);
    br.maxrec = 0;
    br.max_strip_len = 0;
    for (int j = 0; j < n; j++) {
        ShotState &sh = ss->shots[k0 + j];
        Slot &sl = ss->slots[j];
        ShotDev &d = br.hd[j];
        std::memset(&d, 0, sizeof(d));
        d.X = sh.X; d.Z = sh.Z; d.npml = s.npml; d.pitch = sh.pitch;
        d.nxi = sh.nxi; d.nzi = sh.nzi;
        d.nsx = sh.g.nsx; d.nsz = sh.g.nsz;
        d.sbx0 = sh.sbx0; d.sbz0 = sh.sbz0; d.sbnx = sh.sbnx; d.sbnz = sh.sbnz;
        d.rz = sh.g.rz; d.rx0 = sh.g.rx0; d.nrec = sh.g.nrec;
        d.ntx = (sh.X + RTM_BX - 1) / RTM_BX;
        d.strip_len = sh.strip_len;
        d.inv_rho_f = sh.mf.inv_rho; d.kappa_f = sh.mf.kappa;
        d.inv_rho_b = sh.mb.inv_rho; d.kappa_b = sh.mb.kappa;
        d.pml = sh.pml; d.src = sh.src;
        d.a = sl.a; d.b = sl.b;
        d.strips = sl.strips; d.strip_scale = sl.strip_scale; d.strip_stage = sl.strip_stage;
        d.gather = s.mode == 0 ? sh.gather_raw : sh.gather32;
        d.gather_scale = nullptr;
        d.g1 = sl.g1; d.illum = sl.illum;
        d.g1t = sl.g1t; d.illt = sl.illt;
        for (int k = 0; k < 4; k++) d.gx[k] = sl.gx[k];
        d.ps_pre = sl.ps_pre; d.p_pre = sl.p_pre;
        d.vp2_b = sh.mb.vp2;
        // tensor maps of the fields the stencil kernels stage, for this shot's row pitch
        {
            const int vh = ss->bz_vel + RTM_STAGE_ZEXTRA_VEL, ph = ss->bz_pres + RTM_STAGE_ZEXTRA_PRES;
            const int vhr = ss->bz_vel_recon + RTM_STAGE_ZEXTRA_VEL, phr = ss->bz_pres_recon + RTM_STAGE_ZEXTRA_PRES;
            // whole-step kernel: p of both buffers of each wavefield (placeholders when off)
            const int sw = RTM_BX + 48, sh_ = ss->tz_step + 38;
            const WaveDev &A1 = ss->fused ? sl.a2 : sl.a, &B1 = ss->fused ? sl.b2 : sl.b;
            const int tz = ss->tz_step;
            struct { float *f; int w, h; } m[RTM_TMAP_COUNT] = {
                {sl.a.p, RTM_STAGE_W, vh}, {sl.a.vx, RTM_STAGE_W, ss->bz_pres}, {sl.a.vz, RTM_BX, ph},
                {sl.b.p, RTM_STAGE_W, vh}, {sl.b.vx, RTM_STAGE_W, ss->bz_pres}, {sl.b.vz, RTM_BX, ph},
                {sl.a.p, RTM_STAGE_W, vhr}, {sl.a.p, sw, sh_}, {A1.p, sw, sh_}, {sl.b.p, sw, sh_}, {B1.p, sw, sh_},
                {sl.a.vx, RTM_STAGE_W, tz}, {A1.vx, RTM_STAGE_W, tz}, {sl.b.vx, RTM_STAGE_W, tz}, {B1.vx, RTM_STAGE_W, tz},
                {sl.a.vz, RTM_BX, tz + 20}, {A1.vz, RTM_BX, tz + 20}, {sl.b.vz, RTM_BX, tz + 20}, {B1.vz, RTM_BX, tz + 20},
                {sl.a.vx, RTM_STAGE_W, ss->bz_pres_recon}, {sl.a.vz, RTM_BX, phr}};
            for (int t = 0; t < RTM_TMAP_COUNT; t++) {
                CUtensorMap cm;
                int rc = encode_field_map(&cm, m[t].f, sh.pitch, sh.Z, m[t].w, m[t].h);
                if (rc) return rc;
                std::memcpy(&maps[((size_t)j * RTM_TMAP_COUNT + t) * RTM_TMAP_BYTES], &cm, RTM_TMAP_BYTES);
            }
            d.tmaps = (const char *)ss->d_tmaps + (size_t)j * RTM_TMAP_COUNT * RTM_TMAP_BYTES;
        }
        {
            std::vector<TileRef> *L[4] = {&tiles, &tiles_p, &tiles_r, &tiles_pr};
            shot_tiles(ss, sh, j, fast, L);
        }
        br.maxrec = std::max(br.maxrec, sh.g.nrec);
        br.max_strip_len = std::max(br.max_strip_len, sh.strip_len);
        size_t fb = (size_t)sh.pitch * sh.Z * 4;
        float *f[16] = {sl.a.p,  sl.a.vx, sl.a.vz,  sl.a.sx,  sl.a.sz, sl.b.p,   sl.b.vx,  sl.b.vz,
                        sl.b.sx, sl.b.sz, sl.a2.p, sl.a2.vx, sl.a2.vz, sl.b2.p, sl.b2.vx, sl.b2.vz};
        for (int i = 0; i < (ss->fused ? 16 : 10); i++) CK(cudaMemsetAsync(f[i], 0, fb, st));
        const size_t cells = (size_t)sh.pitch * sh.Z, ib = cells * (o.accum_fp64 ? 8 : 4);
        CK(cudaMemsetAsync(sl.g1, 0, cells * acc_bytes(o), st));
        CK(cudaMemsetAsync(sl.illum, 0, cells * acc_bytes(o), st));
        if (sl.g1t) {
            CK(cudaMemsetAsync(sl.g1t, 0, cells * 8, st));
            CK(cudaMemsetAsync(sl.illt, 0, cells * 8, st));
        }
        if (o.extra_images)
            for (void *g : sl.gx) CK(cudaMemsetAsync(g, 0, ib, st));
    }
    {
        // RTM_B200_TILE_ORDER=position: order each list by tile position and then by shot, so
        // the shots that share a model window read its rows back to back (the default order,
        // shot by shot, keeps a shot's neighbouring tiles together instead)
        const char *e = std::getenv("RTM_B200_TILE_ORDER");
        if (e && !std::strcmp(e, "position"))
            for (std::vector<TileRef> *v : {&tiles, &tiles_p, &tiles_r, &tiles_pr})
                std::stable_sort(v->begin(), v->end(), [](const TileRef &a, const TileRef &b) {
                    return a.z0 != b.z0 ? a.z0 < b.z0 : a.x0 < b.x0;
                });
    }
    br.ntiles = (int)tiles.size();
    br.ntiles_p = (int)tiles_p.size();
    br.ntiles_r = (int)tiles_r.size();
    br.ntiles_pr = (int)tiles_pr.size();
    if (std::max(std::max(br.ntiles, br.ntiles_p), std::max(br.ntiles_r, br.ntiles_pr)) > ss->max_tiles)
        return fail(RTM_ERR_ARG, "tile table overflow");
    const int counts[4] = {br.ntiles, br.ntiles_p, br.ntiles_r, br.ntiles_pr};
    CK(cudaMemcpyAsync(ss->d_counts, counts, sizeof(counts), cudaMemcpyHostToDevice, st));
    {   // tiles per shot: source pass lists (velocity, pressure), backward lists (reconstruction
        // velocity and pressure, receiver velocity and pressure)
        std::vector<int> per(6 * (size_t)ss->B, 0);
        const std::vector<TileRef> *L[6] = {&tiles, &tiles_p, &tiles_r, &tiles_pr, &tiles, &tiles_p};
        for (int l = 0; l < 6; l++)
            for (const TileRef &t : *L[l]) per[(size_t)l * ss->B + t.shot]++;
        CK(cudaMemcpyAsync(ss->d_per_shot, per.data(), sizeof(int) * per.size(), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));   // the host vector goes out of scope
    }
    for (int L = 0; L < 4; L++) br.grid[L] = counts[L];
    br.strip_grid = br.max_strip_len;
    for (int j = 0; j < n; j++) {
        br.ex_nxi = std::max(br.ex_nxi, ss->shots[k0 + j].nxi);
        br.ex_nzi = std::max(br.ex_nzi, ss->shots[k0 + j].nzi);
    }
    if (o.use_graph == 2) {
        // use_graph 2: graph replays launch fixed grids, the counts rounded up to four
        // significant bits (at most 12.5% of blocks idle), so batches of nearby sizes share one
        // captured graph (use_graph 1: exact grids, one graph per launch shape)
        auto bucket = [](int v) {
            int e = 0;
            while ((v >> e) >= 16) e++;
            return ((v + (1 << e) - 1) >> e) << e;
        };
        for (int l = 0; l < 4; l++) br.grid[l] = bucket(counts[l]);
        br.strip_grid = bucket(br.strip_grid);
        br.ex_nxi = bucket(br.ex_nxi);
        br.ex_nzi = bucket(br.ex_nzi);
    }
    for (int j = 0; j < n; j++) {
        const Slot &sl = ss->slots[j];
        br.hd[j].an = sl.a2;
        br.hd[j].bn = sl.b2;
    }
    br.pa = br.pb = 0;
    if (int rc = upload_tables(ss, br)) return rc;
    CK(cudaMemcpyAsync(ss->d_tmaps, maps.data(), maps.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ss->d_tiles, tiles.data(), sizeof(TileRef) * br.ntiles, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ss->d_tiles_p, tiles_p.data(), sizeof(TileRef) * br.ntiles_p, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ss->d_tiles_r, tiles_r.data(), sizeof(TileRef) * br.ntiles_r, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ss->d_tiles_pr, tiles_pr.data(), sizeof(TileRef) * br.ntiles_pr, cudaMemcpyHostToDevice, st));
    StepArgs &a = br.a;
    std::memset(&a, 0, sizeof(a));
    a.shots = ss->d_shots;
    a.tiles = ss->d_tiles;
    a.wavelet = ss->wavelet;
    a.coef = ss->coef;
    for (int i = 0; i < 10; i++) a.c10[i] = ss->coef_host[90 + i];
    a.dt = s.dt;
    a.dtx = s.dt / s.dx;   // rtm_model.cu:73-74
    a.dtz = s.dt / s.dz;
    a.strip_prec = o.strip_precision;
    a.gather_prec = RTM_PREC_FP32;
    // the stencil kernels image into fp32 partial sums in the blocked form
    a.accum_fp64 = o.accum_fp64 == RTM_ACC_FP64_BLOCKED ? RTM_ACC_FP32 : o.accum_fp64;
    a.err = ss->d_err;
    {
        // L2 prefetch of the tiles' operand rows: on for batches of 4 shots or more (measured:
        // +4% at 64 shots per launch, -6% at one shot per launch, where few blocks run and the
        // extra instructions are not hidden); RTM_B200_PREFETCH=0 / 1 forces it
        const char *e = std::getenv("RTM_B200_PREFETCH");
        a.prefetch = (e && *e) ? std::atoi(e) != 0 : n >= 4;
    }
    ss->last_batch_n = n;
    ss->last_batch_shots.clear();
    for (int j = 0; j < n; j++) ss->last_batch_shots.push_back(k0 + j);
    return RTM_OK;
}

// The kernel forms as bits (1: four columns per thread) of vel, vel_recon, pres, pres_recon.
static int form_bits(const rtm_session *ss)
{
    return (ss->vec[0] ? 1 : 0) | (ss->vec[1] ? 2 : 0) | (ss->vec[2] ? 4 : 0) | (ss->vec[3] ? 8 : 0);
}

// Stencil launches in the session's kernel form.
static void vel_step(rtm_session *ss, int mode, int bz, const StepArgs &a, int ntiles)
{
    if (ss->vec[mode == RTM_WAVE_RECON ? 1 : 0]) launch_vel4(mode, bz, a, ntiles, ss->stream);
    else launch_vel(mode, bz, a, ntiles, ss->stream);
}
static void pres_step(rtm_session *ss, int mode, int bz, const StepArgs &a, int ntiles, int record)
{
    if (ss->vec[mode == RTM_WAVE_RECON ? 3 : 2]) launch_pres4(mode, bz, a, ntiles, record, ss->stream);
    else launch_pres(mode, bz, a, ntiles, record, ss->stream);
}

// Full-grid pressure update of one step (interior tiles are flagged in the tile list).
static void launch_pres_tiles(rtm_session *ss, BatchRun &br, int mode, int record)
{
    StepArgs &a = br.a;
    a.tiles = ss->d_tiles_p;
    pres_step(ss, mode, ss->bz_pres, a, list_grid(ss, br, a, 1), record);
    ss->launches++;
}

// Progress lines of the reference (rtm_model.cu:324-326, 415-417), one per shot of the batch
// and snapshot, from the device reductions of the pass just queued.
static int print_snapshots(rtm_session *ss, const BatchRun &br, int side, const char *label, int nsteps, int ntsnap)
{
    const int B = ss->B;
    std::vector<unsigned> h((size_t)ss->nsnap * B);
    CK(cudaMemcpyAsync(h.data(), ss->d_absmax + (size_t)side * ss->nsnap * B, sizeof(unsigned) * h.size(),
                       cudaMemcpyDeviceToHost, ss->stream));
    CK(cudaStreamSynchronize(ss->stream));
    std::vector<int> its;
    if (side == 0)
        for (int it = 0; it < nsteps; it += ntsnap) its.push_back(it);
    else
        for (int it = ss->s.nt - 2; it >= 0; it--)
            if (it % ntsnap == 0) its.push_back(it);
    for (int it : its)
        for (int j = 0; j < br.n; j++) {
            float v;
            unsigned bits = h[(size_t)(it / ntsnap) * B + j];
            std::memcpy(&v, &bits, 4);
            std::printf("%s-the current shot: %d\ttime: %f s; wavefield: %.5e\n", label, ss->shots[br.k0 + j].ishot,
                        it * ss->s.dt, v);
        }
    return RTM_OK;
}

// Run `body` (the launches of one pass's time loop) directly, or, with use_graph, as a CUDA
// graph: captured from the session stream the first time a launch shape `key` is met,
// instantiated, kept, and replayed for every later batch of that shape.  A replayed graph
// launches exactly the kernels, grids and arguments that `body` would: the arguments hold the
// session's device tables (shots, tiles, tensor maps), which each batch rewrites in place
// before its passes run, so equal tile counts mean equal launches.  The kernel count of a
// replay is added to the session's launch count.
template <typename F>
static int run_pass(rtm_session *ss, std::vector<long> key, F &&body)
{
    if (!ss->o.use_graph) {
        body();
        CK(cudaGetLastError());
        return RTM_OK;
    }
    auto it = ss->graphs.find(key);
    if (it == ss->graphs.end()) {
        if (ss->graphs.size() >= 32) {   // bound the cache: shapes vary with uneven apertures
            for (auto &kv : ss->graphs) cudaGraphExecDestroy(kv.second.exec);
            ss->graphs.clear();
        }
        const int l0 = ss->launches;
        CK(cudaStreamBeginCapture(ss->stream, cudaStreamCaptureModeThreadLocal));
        ss->capturing = true;
        body();
        ss->capturing = false;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ss->stream, &g);
        if (e != cudaSuccess) return fail(RTM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        rtm_session::GraphEntry ge;
        e = cudaGraphInstantiate(&ge.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(RTM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        ge.launches = ss->launches - l0;
        ss->launches = l0;
        it = ss->graphs.emplace(std::move(key), ge).first;
    }
    CK(cudaGraphLaunch(it->second.exec, ss->stream));
    ss->launches += it->second.launches;
    return RTM_OK;
}

// One persistent launch for a whole pass (dir 0: source pass; 1: backward pass) when the
// session asks for it and the pass has no part outside it (fp16/bf16 strip packing, the other
// imaging conditions, snapshots); *ran tells whether it ran.
static int persistent_pass(rtm_session *ss, BatchRun &br, int dir, int nsteps, bool save, bool record, bool *ran)
{
    *ran = false;
    const rtm_options &o = ss->o;
    if (!ss->persist || ss->nsnap) return RTM_OK;
    if (dir == 0 && save && o.strip_precision != RTM_PREC_FP32) return RTM_OK;
    if (dir == 1 && (o.extra_images || o.accum_fp64 == RTM_ACC_FP64_BLOCKED)) return RTM_OK;
    cudaStream_t st = ss->stream;
    PassArgs P{};
    P.a = br.a;
    P.a.counts = nullptr;
    P.a.shots = ss->d_shots;
    if (dir == 0) {
        P.list[0] = ss->d_tiles, P.len[0] = br.ntiles;
        P.list[1] = ss->d_tiles_p, P.len[1] = br.ntiles_p;
        P.per_shot = ss->d_per_shot;
    } else {
        P.list[0] = ss->d_tiles_r, P.len[0] = br.ntiles_r;
        P.list[1] = ss->d_tiles_pr, P.len[1] = br.ntiles_pr;
        P.list[2] = ss->d_tiles, P.len[2] = br.ntiles;
        P.list[3] = ss->d_tiles_p, P.len[3] = br.ntiles_p;
        P.per_shot = ss->d_per_shot + 2 * (size_t)ss->B;
    }
    P.B = ss->B;
    P.nshots = br.n;
    P.nsteps = dir == 0 ? nsteps : ss->s.nt - 1;
    P.nt = ss->s.nt;
    P.save = save;
    P.record = record;
    P.strip_prec = o.strip_precision;
    P.queue = ss->d_queue;
    P.done = ss->d_done;
    P.wait_ns = ss->pass_wait_ns;
    P.trace = ss->d_trace;
    P.trace_len = ss->trace_len;
    CK(cudaMemsetAsync(ss->d_queue, 0, 2 * sizeof(unsigned), st));
    CK(cudaMemsetAsync(ss->d_done, 0, 4 * sizeof(unsigned) * ss->B, st));
    cudaEvent_t e;
    timing_begin(ss, dir == 0 ? "pass_fwd" : "pass_bwd", 7, &e);
    const bool ok = ss->bz_pres_recon == ss->bz_pres && launch_pass(dir, P, ss->bz_vel, ss->bz_vel_recon, ss->bz_pres, st);
    timing_end(ss, e);
    if (!ok) return RTM_OK;
    ss->launches++;
    *ran = true;
    CK(cudaGetLastError());
    return RTM_OK;
}

// Source pass (rtm_model.cu:322-346): nsteps forward steps with the source added; strips
// saved after every step when `save` (one small copy kernel, so the stencil kernels carry no
// strip logic); the gather recorded when `record` (mode 0 fuses the reference's separate
// modelling pass, rtm_model.cu:266-290, which is the same computation in the same model,
// into this pass).
static int batch_forward(rtm_session *ss, BatchRun &br, int nsteps, bool save, bool record)
{
    const rtm_options &o = ss->o;
    cudaStream_t st = ss->stream;
    StepArgs &a = br.a;
    const int ntsnap = ss->nsnap ? (int)(o.tsnap / ss->s.dt) : 0;
    if (ntsnap) CK(cudaMemsetAsync(ss->d_absmax, 0, sizeof(unsigned) * ss->nsnap * ss->B, st));
    nvtxRangePushA(record && !save ? "rtm: modelling pass" : "rtm: source pass");
    auto loop = [&] {
        for (int it = 0; it < nsteps; it++) {
            a.it = it;
            a.ring = it % kRing;
            const int mode = RTM_WAVE_FWD;
            if (ntsnap && it % ntsnap == 0) {   // rtm_model.cu:324-326: |p| before the step
                launch_absmax(table(ss, br), br.n, 0, ss->d_absmax + (size_t)(it / ntsnap) * ss->B, st);
                ss->launches++;
            }
            cudaEvent_t e;
            if (ss->fused) {   // velocity and pressure in one launch per tile kind; then swap buffers
                timing_begin(ss, "step_fwd", it, &e);
                a.shots = table(ss, br);
                a.tiles = ss->d_tiles;
                launch_step(mode, ss->tz_step, true, a, list_grid(ss, br, a, 0), record ? 1 : 0, st);
                a.tiles = ss->d_tiles_p;
                launch_step(mode, ss->tz_step, false, a, list_grid(ss, br, a, 1), record ? 1 : 0, st);
                timing_end(ss, e);
                ss->launches += 2;
                br.pa ^= 1;
            } else {
                timing_begin(ss, "vel_fwd", it, &e);
                a.tiles = ss->d_tiles;
                vel_step(ss, mode, ss->bz_vel, a, list_grid(ss, br, a, 0));
                timing_end(ss, e);
                timing_begin(ss, "pres_fwd", it, &e);
                launch_pres_tiles(ss, br, mode, record ? 1 : 0);
                timing_end(ss, e);
                ss->launches += 1;
            }
            if (save) {
                timing_begin(ss, "strip_save", it, &e);
                launch_strip_save(table(ss, br), br.n, br.strip_grid, it, a.ring, o.strip_precision, st);
                timing_end(ss, e);
                ss->launches++;
            }
            if (save && o.strip_precision != RTM_PREC_FP32 && (a.ring == kRing - 1 || it == nsteps - 1)) {
                // timed on every 8th ring (the sampling step of timing_begin)
                timing_begin(ss, "strip_pack", (it / kRing) % 8 == 1 ? 7 : 0, &e);
                launch_strip_pack(table(ss, br), br.n, it - a.ring, 0, a.ring + 1, o.strip_precision, st);
                timing_end(ss, e);
                ss->launches++;
            }
        }
    };
    bool ran = false;
    if (int rc = persistent_pass(ss, br, 0, nsteps, save, record, &ran)) {
        nvtxRangePop();
        return rc;
    }
    if (ran) {
        // every step ran in the one persistent launch
    } else if (ntsnap) {   // snapshots read back per pass: no graph
        loop();
        CK(cudaGetLastError());
    } else {
        const int pa0 = br.pa;
        int rc = run_pass(ss, {0, br.n, br.grid[0], br.grid[1], br.strip_grid, nsteps, save, record, ss->bz_vel,
                               ss->bz_pres, form_bits(ss), ss->fused, ss->tz_step, pa0, br.pb}, loop);
        // a replayed graph swaps the buffers as the captured loop did
        if (!rc && ss->fused && ss->o.use_graph) br.pa = pa0 ^ (nsteps & 1);
        if (rc) {
            nvtxRangePop();
            return rc;
        }
    }
    nvtxRangePop();
    if (ntsnap) return print_snapshots(ss, br, 0, save ? "source" : "forward", nsteps, ntsnap);
    return RTM_OK;
}

// With the whole-step kernel the current fields may lie in the second buffers; copy them to
// the first ones, where the readers of a slot's fields look (rtm_session_get_wavefields,
// rtm_forward).
static int settle_fields(rtm_session *ss, BatchRun &br)
{
    if (!ss->fused) return RTM_OK;
    for (int j = 0; j < br.n; j++) {
        const ShotState &sh = ss->shots[br.k0 + j];
        Slot &sl = ss->slots[j];
        const size_t fb = (size_t)sh.pitch * sh.Z * 4;
        const int par[2] = {br.pa, br.pb};
        const WaveDev *from[2] = {&sl.a2, &sl.b2}, *to[2] = {&sl.a, &sl.b};
        for (int w = 0; w < 2; w++)
            if (par[w]) {
                CK(cudaMemcpyAsync(to[w]->p, from[w]->p, fb, cudaMemcpyDeviceToDevice, ss->stream));
                CK(cudaMemcpyAsync(to[w]->vx, from[w]->vx, fb, cudaMemcpyDeviceToDevice, ss->stream));
                CK(cudaMemcpyAsync(to[w]->vz, from[w]->vz, fb, cudaMemcpyDeviceToDevice, ss->stream));
            }
    }
    br.pa = br.pb = 0;
    return RTM_OK;
}

// Backward pass (rtm_model.cu:348-456) and stacking (:458-488).
static int batch_backward(rtm_session *ss, BatchRun &br)
{
    const rtm_survey &s = ss->s;
    const rtm_options &o = ss->o;
    cudaStream_t st = ss->stream;
    const int n = br.n;
    StepArgs &a = br.a;
    for (int j = 0; j < n; j++) {
        ShotState &sh = ss->shots[br.k0 + j];
        if (s.mode == 0) {
            int rc = finish_gather(ss, sh);
            if (rc) return rc;
        } else if (!sh.gather_ready) {
            return fail(RTM_ERR_ARG, "shot " + std::to_string(sh.ishot) + " has no gather (rtm_session_set_gather)");
        }
        if (o.gather_precision != RTM_PREC_FP32) {
            br.hd[j].gather = sh.gather_packed;
            br.hd[j].gather_scale = sh.gather_scale;
        } else {
            br.hd[j].gather = sh.gather32;
        }
    }
    if (int rc = upload_tables(ss, br)) return rc;
    a.gather_prec = o.gather_precision;
    // ps = final forward p; vxs = vzs = 0 (rtm_model.cu:367-372); the receiver wavefield
    // starts from rest with the last gather sample injected (:410)
    for (int j = 0; j < n; j++) {
        ShotState &sh = ss->shots[br.k0 + j];
        Slot &sl = ss->slots[j];
        const WaveDev &ca = br.pa ? sl.a2 : sl.a;   // the current source-side buffer
        size_t fb = (size_t)sh.pitch * sh.Z * 4;
        CK(cudaMemsetAsync(ca.vx, 0, fb, st));
        CK(cudaMemsetAsync(ca.vz, 0, fb, st));
    }
    launch_inject(table(ss, br), n, br.maxrec, s.nt - 1, s.dt, o.gather_precision, st);
    ss->launches++;
    // the other imaging conditions compare each step with the pressures before it
    // (rtm_model.cu:419-420); their kernel keeps ps_pre/p_pre current from then on
    int max_nxi = 0, max_nzi = 0;   // (the launches use br.ex_nxi, br.ex_nzi)
    if (o.extra_images)
        for (int j = 0; j < n; j++) {
            const ShotState &sh = ss->shots[br.k0 + j];
            const Slot &sl = ss->slots[j];
            const size_t fb = (size_t)sh.pitch * sh.Z * 4;
            CK(cudaMemcpyAsync(sl.ps_pre, (br.pa ? sl.a2 : sl.a).p, fb, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(sl.p_pre, (br.pb ? sl.b2 : sl.b).p, fb, cudaMemcpyDeviceToDevice, st));
            max_nxi = std::max(max_nxi, sh.nxi);
            max_nzi = std::max(max_nzi, sh.nzi);
        }
    const int ntsnap = ss->nsnap ? (int)(o.tsnap / s.dt) : 0;
    unsigned *snap_b = ntsnap ? ss->d_absmax + (size_t)ss->nsnap * ss->B : nullptr;
    if (ntsnap) CK(cudaMemsetAsync(snap_b, 0, sizeof(unsigned) * ss->nsnap * ss->B, st));
    nvtxRangePushA("rtm: backward pass");
    // blocked accumulation: the partial sums go into the fp64 totals every RTM_ACC_BLOCK steps
    // and after the last step (it = 0)
    auto flush_images = [&](int it) {
        if (o.accum_fp64 != RTM_ACC_FP64_BLOCKED || it % RTM_ACC_BLOCK) return;
        cudaEvent_t e;
        timing_begin(ss, "image_flush", (it / RTM_ACC_BLOCK) % 4 == 1 ? 7 : 0, &e);   // every 4th flush
        launch_image_flush(table(ss, br), n, br.ex_nxi, br.ex_nzi, st);
        timing_end(ss, e);
        ss->launches++;
    };
    auto loop = [&] {
        for (int it = s.nt - 2; it >= 0; it--) {
            a.it = it;
            cudaEvent_t e;
            if (ntsnap && it % ntsnap == 0) {   // rtm_model.cu:415-417: receiver |p| before the step
                launch_absmax(table(ss, br), n, 1, snap_b + (size_t)(it / ntsnap) * ss->B, st);
                ss->launches++;
            }
            // reconstruction of the source wavefield, then the receiver wavefield and imaging
            // (which reads the reconstructed pressure of the same step)
            if (ss->fused) {
                timing_begin(ss, "step_recon", it, &e);
                a.shots = table(ss, br);
                a.tiles = ss->d_tiles_r;
                launch_step(RTM_WAVE_RECON, ss->tz_step, true, a, list_grid(ss, br, a, 2), 0, st);
                a.tiles = ss->d_tiles_pr;
                launch_step(RTM_WAVE_RECON, ss->tz_step, false, a, list_grid(ss, br, a, 3), 0, st);
                timing_end(ss, e);
                br.pa ^= 1;
                timing_begin(ss, "step_recv", it, &e);
                a.shots = table(ss, br);
                a.tiles = ss->d_tiles;
                launch_step(RTM_WAVE_RECEIVER, ss->tz_step, true, a, list_grid(ss, br, a, 0), 0, st);
                a.tiles = ss->d_tiles_p;
                launch_step(RTM_WAVE_RECEIVER, ss->tz_step, false, a, list_grid(ss, br, a, 1), 0, st);
                timing_end(ss, e);
                br.pb ^= 1;
                ss->launches += 4;
                flush_images(it);
                if (o.extra_images) {
                    launch_image_extra(table(ss, br), n, br.ex_nxi, br.ex_nzi, o.extra_images == 2, o.accum_fp64, s.dx,
                                       s.dz, s.dt, st);
                    ss->launches++;
                }
                continue;
            }
            timing_begin(ss, "vel_recon", it, &e);
            a.tiles = ss->d_tiles_r;
            vel_step(ss, RTM_WAVE_RECON, ss->bz_vel_recon, a, list_grid(ss, br, a, 2));
            timing_end(ss, e);
            timing_begin(ss, "pres_recon", it, &e);
            a.tiles = ss->d_tiles_pr;
            pres_step(ss, RTM_WAVE_RECON, ss->bz_pres_recon, a, list_grid(ss, br, a, 3), 0);
            timing_end(ss, e);
            timing_begin(ss, "vel_recv", it, &e);
            a.tiles = ss->d_tiles;
            vel_step(ss, RTM_WAVE_RECEIVER, ss->bz_vel, a, list_grid(ss, br, a, 0));
            timing_end(ss, e);
            timing_begin(ss, "pres_recv", it, &e);
            launch_pres_tiles(ss, br, RTM_WAVE_RECEIVER, 0);
            timing_end(ss, e);
            ss->launches += 3;
            flush_images(it);
            if (o.extra_images) {
                launch_image_extra(ss->d_shots, n, br.ex_nxi, br.ex_nzi, o.extra_images == 2, o.accum_fp64, s.dx, s.dz,
                                   s.dt, st);
                ss->launches++;
            }
        }
    };
    bool ran = false;
    if (int rc = persistent_pass(ss, br, 1, s.nt - 1, false, false, &ran)) {
        nvtxRangePop();
        return rc;
    }
    if (ran) {
        // every step ran in the one persistent launch
    } else if (ntsnap) {
        loop();
        CK(cudaGetLastError());
    } else {
        const int pa0 = br.pa, pb0 = br.pb;
        int rc = run_pass(ss, {1, n, br.grid[0], br.grid[1], br.grid[2], br.grid[3], br.ex_nxi, br.ex_nzi,
                               a.gather_prec, ss->bz_vel, ss->bz_vel_recon, ss->bz_pres, ss->bz_pres_recon,
                               form_bits(ss), ss->fused, ss->tz_step, pa0, pb0}, loop);
        if (!rc && ss->fused && ss->o.use_graph) {   // a replayed graph swaps as the captured loop did
            br.pa = pa0 ^ ((s.nt - 1) & 1);
            br.pb = pb0 ^ ((s.nt - 1) & 1);
        }
        if (rc) {
            nvtxRangePop();
            return rc;
        }
    }
    nvtxRangePop();
    if (ntsnap) {
        int rc = print_snapshots(ss, br, 1, "backward", s.nt, ntsnap);
        if (rc) return rc;
    }
    if (int rc = settle_fields(ss, br)) return rc;
    nvtxRangePushA("rtm: stacking");
    std::vector<char> fin(finalize_shot_size() * n);
    for (int j = 0; j < n; j++) {
        ShotState &sh = ss->shots[br.k0 + j];
        int nwin = 50;   // rtm_model.cu:70, :464-465
        while (2 * nwin >= sh.nxi) nwin -= 3;
        const Slot &sl = ss->slots[j];
        const bool blocked = o.accum_fp64 == RTM_ACC_FP64_BLOCKED;   // the totals hold every step
        fill_finalize_shot(fin.data() + j * finalize_shot_size(), blocked ? (void *)sl.g1t : sl.g1,
                           blocked ? (void *)sl.illt : sl.illum, o.extra_images ? sl.gx : nullptr, sh.g.nx1, sh.nxi,
                           nwin, sh.pitch, s.npml, blocked ? RTM_ACC_FP64 : o.accum_fp64);
    }
    CK(cudaMemcpyAsync(ss->d_fin, fin.data(), fin.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(ss->d_nonfinite, 0x7f, sizeof(int), st));   // 0x7f7f7f7f: none
    launch_finalize(ss->d_fin, n, s.nx, s.nz, o.accum_fp64, ss->img1, ss->img2s, ss->img2m, ss->illum,
                    ss->d_nonfinite, st);
    ss->launches++;
    if (o.extra_images) {
        launch_finalize_extra(ss->d_fin, n, s.nx, s.nz, o.accum_fp64, ss->ximg, st);
        ss->launches++;
    }
    nvtxRangePop();
    CK(cudaGetLastError());
    return RTM_OK;
}

// ---- tile-height and kernel-form tuner ------------------------------------------------
// The split stencil kernels take 8-, 16- or 32-row tiles in two forms (one column per thread;
// four columns by U rows per thread); which is fastest depends on the grid (partial tiles, the
// share of PML-band and edge tiles), on the shots per launch (blocks to fill 148 SMs) and on
// the kernel.  Before the first batch of a launch shape, every (height, form) is timed on that
// batch's own buffers: two untimed and four timed source-pass steps (velocity and pressure)
// and backward steps (reconstruction and receiver pass) with CUDA events per kernel, no strips
// saved.  Forward/receiver velocity, reconstruction velocity and reconstruction pressure each
// keep their fastest pair; the forward and receiver pressure kernels share one height (one
// tile list), each taking its faster form at it.  The batch is set up again afterwards, so
// the trial steps leave nothing behind; heights and forms do not change the results (tested
// bit for bit).  Choices are kept per process by launch shape and, with
// RTM_B200_TUNE_CACHE=<file>, in that file ("key vel vel_recon pres pres_recon forms" lines,
// forms a bit set of vel, vel_recon, pres, pres_recon) across processes.  The whole-step kernel's tile
// height is chosen the same way (tune_step_height).
namespace {
std::mutex g_tune_mu;
std::map<std::string, std::array<int, 5>> g_tune;
bool g_tune_loaded = false;
}  // namespace

static std::string tune_key(rtm_session *ss, int k0, int n)
{
    int xmax = 0;
    for (int j = 0; j < n; j++) xmax = std::max(xmax, ss->shots[k0 + j].X);
    char b[200];
    std::snprintf(b, sizeof b, "%s/X%d/Z%d/npml%d/n%d/strip%d/gather%d/acc%d/extra%d/mode%d",
                  ss->fused ? "step" : ss->forms_fixed ? (ss->vec[0] ? "vector" : "scalar") : "split",
                  xmax, ss->shots[k0].Z, ss->s.npml, n, ss->o.strip_precision, ss->o.gather_precision, ss->o.accum_fp64,
                  ss->o.extra_images, ss->s.mode);
    return b;
}

// The whole-step kernel's tile height (16 or 32 rows), timed the same way: source-pass,
// reconstruction and receiver steps, each kind's fast and general launches together.  The
// choice is recorded as "key tz tz tz tz 0".
static int tune_step_height(rtm_session *ss, int k0, int n, const std::string &key, const char *path)
{
    const int cand[2] = {16, 32};
    double ms[2] = {0, 0};
    cudaEvent_t ev[2][4];
    for (auto &b : ev)
        for (auto &e : b) CK(cudaEventCreate(&e));
    cudaStream_t st = ss->stream;
    int rc = RTM_OK;
    const int steps = 6, warm = 2;
    for (int c = 0; c < 2 && rc == RTM_OK; c++) {
        ss->tz_step = cand[c];
        BatchRun br;
        if ((rc = batch_setup(ss, k0, n, br))) break;
        StepArgs a = br.a;
        for (int it = 0; it < steps; it++) {
            const int t = it - warm;
            a.it = std::min(it + 1, ss->s.nt - 2);
            if (t >= 0) cudaEventRecord(ev[0][t], st);
            const int modes[3] = {RTM_WAVE_FWD, RTM_WAVE_RECON, RTM_WAVE_RECEIVER};
            for (int m : modes) {
                a.shots = table(ss, br);
                const bool recon = m == RTM_WAVE_RECON;
                a.tiles = recon ? ss->d_tiles_r : ss->d_tiles;
                launch_step(m, ss->tz_step, true, a, recon ? br.ntiles_r : br.ntiles, 0, st);
                a.tiles = recon ? ss->d_tiles_pr : ss->d_tiles_p;
                launch_step(m, ss->tz_step, false, a, recon ? br.ntiles_pr : br.ntiles_p, 0, st);
                if (m == RTM_WAVE_RECEIVER) br.pb ^= 1;
                else br.pa ^= 1;
            }
            if (t >= 0) cudaEventRecord(ev[1][t], st);
        }
        ss->launches += 6 * steps;
        if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = fail(RTM_ERR_CUDA, "tile-height trial launches failed");
            break;
        }
        for (int t = 0; t < steps - warm; t++) {
            float m = 0.f;
            cudaEventElapsedTime(&m, ev[0][t], ev[1][t]);
            ms[c] += m;
        }
    }
    for (auto &b : ev)
        for (auto &e : b) cudaEventDestroy(e);
    if (rc) return rc;
    if ((rc = check_kernel_flag(ss))) return rc;
    const int tz = ms[0] < ms[1] ? cand[0] : cand[1];
    ss->tz_step = tz;
    if (ss->o.verbose)
        std::printf("rtm_b200: step tile height for %s: %d (ms per 4 steps: 16 rows %.3f, 32 rows %.3f)\n", key.c_str(),
                    tz, ms[0], ms[1]);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = {tz, tz, tz, tz, 0};
    if (path && *path)
        if (FILE *f = std::fopen(path, "a")) {
            std::fprintf(f, "%s %d %d %d %d 0\n", key.c_str(), tz, tz, tz, tz);
            std::fclose(f);
        }
    return RTM_OK;
}

static int tune_heights(rtm_session *ss, int k0, int n)
{
    if (!ss->tune) return RTM_OK;
    const std::string key = tune_key(ss, k0, n);
    const char *path = std::getenv("RTM_B200_TUNE_CACHE");
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        if (!g_tune_loaded && path && *path) {
            g_tune_loaded = true;
            if (FILE *f = std::fopen(path, "r")) {
                char k[200];
                int v[5];
                while (std::fscanf(f, "%199s %d %d %d %d %d", k, &v[0], &v[1], &v[2], &v[3], &v[4]) == 6)
                    g_tune[k] = {v[0], v[1], v[2], v[3], v[4]};
                std::fclose(f);
            }
        }
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            if (ss->fused) {
                ss->tz_step = it->second[0];
                return RTM_OK;
            }
            ss->bz_vel = it->second[0];
            ss->bz_vel_recon = it->second[1];
            ss->bz_pres = it->second[2];
            ss->bz_pres_recon = it->second[3];
            for (int f = 0; f < 4; f++) ss->vec[f] = (it->second[4] >> f) & 1;
            return RTM_OK;
        }
    }
    if (ss->fused) return tune_step_height(ss, k0, n, key, path);
    // candidates: tile height x kernel form (both forms unless RTM_B200_KERNELS fixes one)
    std::vector<std::pair<int, int>> cand;   // (bz, vector form)
    for (int bz : {8, 16, 32})
        for (int f = 0; f < 2; f++)
            if (!ss->forms_fixed || f == (ss->vec[0] ? 1 : 0)) cand.push_back({bz, f});
    const int nc = (int)cand.size();
    const char *names[6] = {"vel_fwd", "pres_fwd", "vel_recon", "pres_recon", "vel_recv", "pres_recv"};
    std::vector<std::array<double, 6>> ms(nc, std::array<double, 6>{});
    cudaEvent_t ev[2][6][4];
    for (auto &a : ev)
        for (auto &b : a)
            for (auto &e : b) CK(cudaEventCreate(&e));
    cudaStream_t st = ss->stream;
    int rc = RTM_OK;
    const int steps = 6, warm = 2;
    for (int c = 0; c < nc && rc == RTM_OK; c++) {
        ss->bz_vel = ss->bz_vel_recon = ss->bz_pres = ss->bz_pres_recon = cand[c].first;
        for (bool &v : ss->vec) v = cand[c].second != 0;
        BatchRun br;
        if ((rc = batch_setup(ss, k0, n, br))) break;
        StepArgs a = br.a;
        for (int it = 0; it < steps; it++) {
            const int t = it - warm;
            a.it = std::min(it + 1, ss->s.nt - 2);
            auto rec = [&](int k, int side) {
                if (t >= 0) cudaEventRecord(ev[side][k][t], st);
            };
            rec(0, 0); a.tiles = ss->d_tiles; vel_step(ss, RTM_WAVE_FWD, ss->bz_vel, a, br.ntiles); rec(0, 1);
            rec(1, 0); a.tiles = ss->d_tiles_p; pres_step(ss, RTM_WAVE_FWD, ss->bz_pres, a, br.ntiles_p, 0); rec(1, 1);
            rec(2, 0); a.tiles = ss->d_tiles_r; vel_step(ss, RTM_WAVE_RECON, ss->bz_vel_recon, a, br.ntiles_r); rec(2, 1);
            rec(3, 0); a.tiles = ss->d_tiles_pr; pres_step(ss, RTM_WAVE_RECON, ss->bz_pres_recon, a, br.ntiles_pr, 0);
            rec(3, 1);
            rec(4, 0); a.tiles = ss->d_tiles; vel_step(ss, RTM_WAVE_RECEIVER, ss->bz_vel, a, br.ntiles); rec(4, 1);
            rec(5, 0); a.tiles = ss->d_tiles_p; pres_step(ss, RTM_WAVE_RECEIVER, ss->bz_pres, a, br.ntiles_p, 0); rec(5, 1);
        }
        ss->launches += 6 * steps;
        if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = fail(RTM_ERR_CUDA, "tile-height trial launches failed");
            break;
        }
        for (int k = 0; k < 6; k++)
            for (int t = 0; t < steps - warm; t++) {
                float m = 0.f;
                cudaEventElapsedTime(&m, ev[0][k][t], ev[1][k][t]);
                ms[c][k] += m;
            }
    }
    for (auto &a : ev)
        for (auto &b : a)
            for (auto &e : b) cudaEventDestroy(e);
    if (rc) return rc;
    if ((rc = check_kernel_flag(ss))) return rc;
    // the fastest (height, form) of each family, the forward and receiver kernels of a field
    // together (they share a tile list and a form)
    auto argmin = [&](auto cost) {
        int bi = 0;
        for (int c = 1; c < nc; c++)
            if (cost(c) < cost(bi)) bi = c;
        return bi;
    };
    const int cv = argmin([&](int c) { return ms[c][0] + ms[c][4]; });
    const int cr = argmin([&](int c) { return ms[c][2]; });
    const int cp = argmin([&](int c) { return ms[c][1] + ms[c][5]; });
    const int cpr = argmin([&](int c) { return ms[c][3]; });
    ss->bz_vel = cand[cv].first;
    ss->bz_vel_recon = cand[cr].first;
    ss->bz_pres = cand[cp].first;
    ss->bz_pres_recon = cand[cpr].first;
    ss->vec[0] = cand[cv].second;
    ss->vec[1] = cand[cr].second;
    ss->vec[2] = cand[cp].second;
    ss->vec[3] = cand[cpr].second;
    const std::array<int, 5> pick = {ss->bz_vel, ss->bz_vel_recon, ss->bz_pres, ss->bz_pres_recon, form_bits(ss)};
    if (ss->o.verbose) {
        std::printf("rtm_b200: tiles for %s: vel %d%s, vel_recon %d%s, pres %d%s, pres_recon %d%s (ms per 4 steps:",
                    key.c_str(), pick[0], ss->vec[0] ? "v" : "s", pick[1], ss->vec[1] ? "v" : "s", pick[2],
                    ss->vec[2] ? "v" : "s", pick[3], ss->vec[3] ? "v" : "s");
        for (int c = 0; c < nc; c++)
            for (int k = 0; k < 6; k++)
                std::printf(" %s@%d%s=%.3f", names[k], cand[c].first, cand[c].second ? "v" : "s", ms[c][k]);
        std::printf(")\n");
    }
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = pick;
    if (path && *path)
        if (FILE *f = std::fopen(path, "a")) {
            std::fprintf(f, "%s %d %d %d %d %d\n", key.c_str(), pick[0], pick[1], pick[2], pick[3], pick[4]);
            std::fclose(f);
        }
    return RTM_OK;
}

static int run_batch(rtm_session *ss, int k0, int n)
{
    BatchRun br;
    int rc = tune_heights(ss, k0, n);
    if (rc) return rc;
    rc = batch_setup(ss, k0, n, br);
    if (rc) return rc;
    nvtxRangePushA("rtm: batch");
    if (!(rc = batch_forward(ss, br, ss->s.nt, true, ss->s.mode == 0))) rc = batch_backward(ss, br);
    nvtxRangePop();
    if (rc) return rc;
    CK(cudaStreamSynchronize(ss->stream));
    if ((rc = check_kernel_flag(ss))) return rc;
    if ((rc = check_guards(ss))) return rc;
    return check_nonfinite(ss, k0, n);
}

int session_batch_size(rtm_session *ss) { return ss ? ss->B : 0; }

// Shots in the next launch of a run over `remaining` shots: the run is split into
// ceil(remaining / B) launches of equal size (to within one shot), so that no launch is a
// small remainder that leaves most of the SMs idle for a whole pass (256 shots with room for
// 246: two launches of 128, not 246 and 10).
int session_wave_size(const rtm_session *ss, int remaining)
{
    const int waves = (remaining + ss->B - 1) / ss->B;
    return (remaining + waves - 1) / waves;
}

// Choose the kernel configuration of every launch shape of a run over shots [k0, k0+n) now
// (the tuner's trial steps), so that a timed run does not include them.
int session_prepare(rtm_session *ss, int k0, int n)
{
    if (!ss || k0 < 0 || n < 1 || k0 + n > (int)ss->shots.size()) return fail(RTM_ERR_ARG, "bad shot range");
    CK(cudaSetDevice(ss->dev));
    for (int b0 = k0; b0 < k0 + n;) {
        const int m = session_wave_size(ss, k0 + n - b0);
        if (int rc = tune_heights(ss, b0, m)) return rc;
        b0 += m;
    }
    CK(cudaStreamSynchronize(ss->stream));
    return RTM_OK;
}

// Modelling only (the reference's mode-0 modelling pass, rtm_model.cu:266-290): record
// the gathers of shots [k0, k0+n) without saving strips or migrating.
static int model_range(rtm_session *ss, int k0, int n)
{
    BatchRun br;
    int rc = batch_setup(ss, k0, n, br);
    if (rc) return rc;
    if ((rc = batch_forward(ss, br, ss->s.nt, false, true))) return rc;
    CK(cudaStreamSynchronize(ss->stream));
    if ((rc = check_kernel_flag(ss))) return rc;
    return check_guards(ss);
}

// Run shots [k0, k0+n) (n <= batch size) as one batch.
int session_run_range(rtm_session *ss, int k0, int n)
{
    if (!ss || k0 < 0 || n < 1 || n > ss->B || k0 + n > (int)ss->shots.size())
        return fail(RTM_ERR_ARG, "bad shot range");
    CK(cudaSetDevice(ss->dev));
    return run_batch(ss, k0, n);
}

}  // namespace rtm

using namespace rtm;

extern "C" {

const char *rtm_last_error(void) { return rtm::last_error(); }
const char *rtm_version(void) { return "rtm_b200 0.1 (sm_100a)"; }

int rtm_session_open(rtm_session **out, const rtm_survey *s, const rtm_options *o, const int *shots, int nshots,
                     const float *vp, const float *rho, const float *vp_mig, const float *rho_mig,
                     const float *diffcoef)
{
    clear_error();
    if (!out || !s || !o || !shots || !vp || !rho) return fail(RTM_ERR_ARG, "null argument");
    *out = nullptr;
    rtm_session *ss = new rtm_session();
    ss->s = *s;
    ss->o = *o;
    int rc = open_session(ss, vp, rho, vp_mig, rho_mig, diffcoef, shots, nshots);
    if (rc) {
        rtm_session_close(ss);
        return rc;
    }
    *out = ss;
    return RTM_OK;
}

int rtm_session_open_geometry(rtm_session **out, const rtm_survey *s, const rtm_options *o, const int *shots,
                              const rtm_geometry *geoms, int nshots, const float *vp, const float *rho,
                              const float *vp_mig, const float *rho_mig, const float *diffcoef)
{
    clear_error();
    if (!out || !s || !o || !shots || !geoms || !vp || !rho) return fail(RTM_ERR_ARG, "null argument");
    *out = nullptr;
    rtm_session *ss = new rtm_session();
    ss->s = *s;
    ss->o = *o;
    int rc = open_session(ss, vp, rho, vp_mig, rho_mig, diffcoef, shots, nshots, geoms);
    if (rc) {
        rtm_session_close(ss);
        return rc;
    }
    *out = ss;
    return RTM_OK;
}

int rtm_session_set_gather_raw(rtm_session *ss, int k, const float *seisobs, int nx0, int nt0, float dt0,
                               int mirror)
{
    if (!ss || k < 0 || k >= (int)ss->shots.size() || !seisobs) return fail(RTM_ERR_ARG, "bad gather argument");
    if (mirror != 0 && mirror != 1) return fail(RTM_ERR_ARG, "mirror must be 0 or 1");
    if (ss->s.mode != 1) return fail(RTM_ERR_ARG, "recorded gathers need a mode-1 session");
    ShotState &sh = ss->shots[k];
    CK(cudaSetDevice(ss->dev));
    int nl = 0;
    int rc = interp_gather_device(ss->interp, seisobs, nx0, nt0, sh.gather32, sh.g.nrec, ss->s.nt, ss->s.dt, dt0,
                                  mirror, ss->stream, &nl);
    if (rc) return rc;
    ss->launches += nl;
    rc = finish_gather(ss, sh);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ss->stream));
    if ((rc = interp_check_guards(ss->interp))) return rc;
    return check_guards(ss);
}

int rtm_session_set_gather(rtm_session *ss, int k, const float *gather)
{
    if (!ss || k < 0 || k >= (int)ss->shots.size() || !gather) return fail(RTM_ERR_ARG, "bad gather argument");
    ShotState &sh = ss->shots[k];
    CK(cudaSetDevice(ss->dev));
    CK(cudaMemcpyAsync(sh.gather32, gather, sizeof(float) * (size_t)ss->s.nt * sh.g.nrec, cudaMemcpyHostToDevice,
                       ss->stream));
    int rc = finish_gather(ss, sh);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ss->stream));
    return RTM_OK;
}

int rtm_session_run(rtm_session *ss, rtm_stats *stats)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    CK(cudaSetDevice(ss->dev));
    for (auto &kv : ss->timing) kv.second.used = 0;
    int l0 = ss->launches;
    auto t0 = std::chrono::steady_clock::now();
    int nb = 0;
    double cells = 0;
    for (int k0 = 0; k0 < (int)ss->shots.size();) {
        const int n = session_wave_size(ss, (int)ss->shots.size() - k0);
        int rc = run_batch(ss, k0, n);
        if (rc) return rc;
        nb++;
        for (int j = 0; j < n; j++) {
            const ShotState &sh = ss->shots[k0 + j];
            cells += (double)ss->s.nt * (2.0 * sh.X * sh.Z + (double)sh.nxi * sh.nzi);
        }
        if (ss->o.verbose)
            std::printf("rtm_b200: batch of %d shots done (%d/%zu)\n", n, k0 + n, ss->shots.size());
        k0 += n;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (stats) {
        stats->seconds_total = std::chrono::duration<double>(t1 - t0).count();
        stats->gcell_updates = cells * 1e-9;
        stats->shots = (int)ss->shots.size();
        stats->batches = nb;
        stats->kernel_launches = ss->launches - l0;
    }
    return RTM_OK;
}

int rtm_session_run_range(rtm_session *ss, int k0, int n, rtm_stats *stats)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    if (k0 < 0 || n < 1 || k0 + n > (int)ss->shots.size()) return fail(RTM_ERR_ARG, "bad shot range");
    CK(cudaSetDevice(ss->dev));
    for (auto &kv : ss->timing) kv.second.used = 0;
    int l0 = ss->launches;
    auto t0 = std::chrono::steady_clock::now();
    int nb = 0;
    double cells = 0;
    for (int b0 = k0; b0 < k0 + n;) {
        const int m = session_wave_size(ss, k0 + n - b0);
        int rc = run_batch(ss, b0, m);
        if (rc) return rc;
        nb++;
        for (int j = 0; j < m; j++) {
            const ShotState &sh = ss->shots[b0 + j];
            cells += (double)ss->s.nt * (2.0 * sh.X * sh.Z + (double)sh.nxi * sh.nzi);
        }
        b0 += m;
    }
    if (stats) {
        stats->seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        stats->gcell_updates = cells * 1e-9;
        stats->shots = n;
        stats->batches = nb;
        stats->kernel_launches = ss->launches - l0;
    }
    return RTM_OK;
}

int rtm_session_model(rtm_session *ss)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    if (ss->s.mode != 0) return fail(RTM_ERR_ARG, "modelling needs a mode-0 session");
    CK(cudaSetDevice(ss->dev));
    for (int k0 = 0; k0 < (int)ss->shots.size();) {
        const int n = session_wave_size(ss, (int)ss->shots.size() - k0);
        int rc = model_range(ss, k0, n);
        if (rc) return rc;
        k0 += n;
    }
    return RTM_OK;
}

int rtm_session_image_ptrs(rtm_session *ss, void **image1, void **image2s, void **image2m, void **illum)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    if (image1) *image1 = ss->img1;
    if (image2s) *image2s = ss->img2s;
    if (image2m) *image2m = ss->img2m;
    if (illum) *illum = ss->illum;
    return RTM_OK;
}

int rtm_session_get_gather(rtm_session *ss, int k, float *gather)
{
    if (!ss || k < 0 || k >= (int)ss->shots.size() || !gather) return fail(RTM_ERR_ARG, "bad gather argument");
    const ShotState &sh = ss->shots[k];
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    const float *src = ss->s.mode == 0 ? sh.gather_raw : sh.gather32;
    CK(cudaMemcpy(gather, src, sizeof(float) * (size_t)ss->s.nt * sh.g.nrec, cudaMemcpyDeviceToHost));
    return RTM_OK;
}

int rtm_session_get_pml(rtm_session *ss, int k, float *ddx, float *ddz, float *ddxvx, float *ddzvz)
{
    if (!ss || k < 0 || k >= (int)ss->shots.size()) return fail(RTM_ERR_ARG, "bad shot index");
    const ShotState &sh = ss->shots[k];
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    const PmlOffsets o = pml_offsets(sh.X, sh.Z);
    struct { float *out; int off, n; } part[4] = {
        {ddx, o.ddx, sh.X}, {ddz, o.ddz, sh.Z}, {ddxvx, o.ddxvx, sh.X - 1}, {ddzvz, o.ddzvz, sh.Z - 1}};
    for (const auto &q : part)
        if (q.out) CK(cudaMemcpy(q.out, sh.pml + q.off, sizeof(float) * q.n, cudaMemcpyDeviceToHost));
    return RTM_OK;
}

int rtm_session_prepare(rtm_session *ss, int k0, int n) { return session_prepare(ss, k0, n); }

int rtm_session_batch_size(rtm_session *ss) { return session_batch_size(ss); }

int rtm_session_tile_heights(rtm_session *ss, int *bz_vel, int *bz_vel_recon, int *bz_pres, int *bz_pres_recon)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    if (bz_vel) *bz_vel = ss->fused ? ss->tz_step : ss->bz_vel;
    if (bz_vel_recon) *bz_vel_recon = ss->fused ? ss->tz_step : ss->bz_vel_recon;
    if (bz_pres) *bz_pres = ss->fused ? ss->tz_step : ss->bz_pres;
    if (bz_pres_recon) *bz_pres_recon = ss->fused ? ss->tz_step : ss->bz_pres_recon;
    return RTM_OK;
}

int rtm_session_nrec(rtm_session *ss, int k)
{
    if (!ss || k < 0 || k >= (int)ss->shots.size()) return -1;
    return ss->shots[k].g.nrec;
}

static int copy_image(rtm_session *ss, void *dev, float *out)
{
    if (!out) return RTM_OK;
    size_t n = (size_t)ss->s.nx * ss->s.nz;
    if (ss->o.accum_fp64) {
        std::vector<double> t(n);
        CK(cudaMemcpy(t.data(), dev, n * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; i++) out[i] = (float)t[i];
    } else {
        CK(cudaMemcpy(out, dev, n * 4, cudaMemcpyDeviceToHost));
    }
    return RTM_OK;
}

int rtm_session_get_images(rtm_session *ss, float *image1, float *image2s, float *image2m, float *illum)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    int rc;
    if ((rc = copy_image(ss, ss->img1, image1))) return rc;
    if ((rc = copy_image(ss, ss->img2s, image2s))) return rc;
    if ((rc = copy_image(ss, ss->img2m, image2m))) return rc;
    if ((rc = copy_image(ss, ss->illum, illum))) return rc;
    return RTM_OK;
}

int rtm_session_get_images_f64(rtm_session *ss, double *image1, double *image2s, double *illum)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    if (!ss->o.accum_fp64) return fail(RTM_ERR_ARG, "session accumulates in fp32");
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    size_t n = (size_t)ss->s.nx * ss->s.nz * 8;
    if (image1) CK(cudaMemcpy(image1, ss->img1, n, cudaMemcpyDeviceToHost));
    if (image2s) CK(cudaMemcpy(image2s, ss->img2s, n, cudaMemcpyDeviceToHost));
    if (illum) CK(cudaMemcpy(illum, ss->illum, n, cudaMemcpyDeviceToHost));
    return RTM_OK;
}

int rtm_session_get_images_extra(rtm_session *ss, float *image3s, float *image4s, float *image5s, float *image3m,
                                 float *image4m, float *image5m, float *imagetrue)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    if (!ss->o.extra_images) return fail(RTM_ERR_ARG, "the session was opened without extra_images");
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    float *out[7] = {image3s, image4s, image5s, image3m, image4m, image5m, imagetrue};
    for (int k = 0; k < 7; k++) {
        int rc = copy_image(ss, ss->ximg[k], out[k]);
        if (rc) return rc;
    }
    return RTM_OK;
}

// ---- checkpoints ----------------------------------------------------------------------
// File: the header below, then the session's stacked images as accumulated (image1, image2s,
// image2m, illum, then with extra_images image3s..5s, image3m..5m, imagetrue), each nx*nz
// elements of elem_bytes (4 or 8).  Written to "<path>.tmp" and renamed over <path>.
struct CheckpointHeader {
    char magic[8];                 // "RTMB200C"
    unsigned version;              // 1
    unsigned elem_bytes;
    unsigned long long config_hash;
    int nx, nz, nshots, shots_done, nimages, batch;
};

static int checkpoint_images(rtm_session *ss, void **img)
{
    int k = 0;
    img[k++] = ss->img1;
    img[k++] = ss->img2s;
    img[k++] = ss->img2m;
    img[k++] = ss->illum;
    if (ss->o.extra_images)
        for (void *x : ss->ximg) img[k++] = x;
    return k;
}

int rtm_session_save_checkpoint(rtm_session *ss, const char *path, int shots_done)
{
    if (!ss || !path) return fail(RTM_ERR_ARG, "null argument");
    if (shots_done < 0 || shots_done > (int)ss->shots.size()) return fail(RTM_ERR_ARG, "shots_done out of range");
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    void *img[11];
    CheckpointHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "RTMB200C", 8);
    h.version = 1;
    h.elem_bytes = ss->o.accum_fp64 ? 8 : 4;
    h.config_hash = ss->config_hash;
    h.nx = ss->s.nx;
    h.nz = ss->s.nz;
    h.nshots = (int)ss->shots.size();
    h.shots_done = shots_done;
    h.nimages = checkpoint_images(ss, img);
    h.batch = ss->B;
    const size_t bytes = (size_t)h.nx * h.nz * h.elem_bytes;
    std::vector<char> buf(bytes);
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return fail(RTM_ERR_IO, "cannot create " + tmp);
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    for (int k = 0; k < h.nimages && ok; k++) {
        if (cudaMemcpy(buf.data(), img[k], bytes, cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
        ok = ok && std::fwrite(buf.data(), 1, bytes, f) == bytes;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return fail(RTM_ERR_IO, std::string("cannot write checkpoint ") + path);
    }
    return RTM_OK;
}

// Reads and checks a checkpoint header (no device work).
static int read_checkpoint_header(const char *path, CheckpointHeader &h, FILE **keep)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot open checkpoint ") + path);
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, "RTMB200C", 8) != 0 || h.version != 1 ||
        (h.elem_bytes != 4 && h.elem_bytes != 8) || h.nx < 1 || h.nz < 1 || h.nimages < 4 || h.nimages > 11 ||
        h.shots_done < 0 || h.shots_done > h.nshots) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("not a checkpoint of this library: ") + path);
    }
    std::fseek(f, 0, SEEK_END);
    const long long want = (long long)sizeof(h) + (long long)h.nimages * h.nx * h.nz * h.elem_bytes;
    if (std::ftell(f) != want) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("truncated checkpoint: ") + path);
    }
    if (keep) {
        std::fseek(f, (long)sizeof(h), SEEK_SET);
        *keep = f;
    } else {
        std::fclose(f);
    }
    return RTM_OK;
}

int rtm_session_load_checkpoint(rtm_session *ss, const char *path, int *shots_done)
{
    if (!ss || !path) return fail(RTM_ERR_ARG, "null argument");
    CheckpointHeader h;
    FILE *f = nullptr;
    int rc = read_checkpoint_header(path, h, &f);
    if (rc) return rc;
    void *img[11];
    const int nimg = checkpoint_images(ss, img);
    if (h.config_hash != ss->config_hash || h.nx != ss->s.nx || h.nz != ss->s.nz ||
        h.nshots != (int)ss->shots.size() || h.nimages != nimg || h.elem_bytes != (ss->o.accum_fp64 ? 8u : 4u)) {
        std::fclose(f);
        return fail(RTM_ERR_ARG, std::string("checkpoint ") + path +
                                     " was written by a run with another survey, model, shot list or image options");
    }
    CK(cudaSetDevice(ss->dev));
    CK(cudaStreamSynchronize(ss->stream));
    const size_t bytes = (size_t)h.nx * h.nz * h.elem_bytes;
    std::vector<char> buf(bytes);
    for (int k = 0; k < nimg && !rc; k++) {
        if (std::fread(buf.data(), 1, bytes, f) != bytes) rc = fail(RTM_ERR_IO, std::string("cannot read ") + path);
        else if (cudaMemcpy(img[k], buf.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(RTM_ERR_CUDA, "checkpoint upload failed");
    }
    std::fclose(f);
    if (!rc && shots_done) *shots_done = h.shots_done;
    return rc;
}

int rtm_checkpoint_info(const char *path, int *nx, int *nz, int *nshots, int *shots_done, int *elem_bytes,
                        unsigned long long *config_hash)
{
    clear_error();
    if (!path) return fail(RTM_ERR_ARG, "null path");
    CheckpointHeader h;
    int rc = read_checkpoint_header(path, h, nullptr);
    if (rc) return rc;
    if (nx) *nx = h.nx;
    if (nz) *nz = h.nz;
    if (nshots) *nshots = h.nshots;
    if (shots_done) *shots_done = h.shots_done;
    if (elem_bytes) *elem_bytes = (int)h.elem_bytes;
    if (config_hash) *config_hash = h.config_hash;
    return RTM_OK;
}

unsigned long long rtm_session_config_hash(rtm_session *ss) { return ss ? ss->config_hash : 0ULL; }

int rtm_session_guard_count(rtm_session *ss) { return session_guard_count(ss); }

int rtm_session_reset_images(rtm_session *ss)
{
    if (!ss) return fail(RTM_ERR_ARG, "null session");
    size_t isz = (size_t)ss->s.nx * ss->s.nz * (ss->o.accum_fp64 ? 8 : 4);
    CK(cudaMemsetAsync(ss->img1, 0, isz, ss->stream));
    CK(cudaMemsetAsync(ss->img2s, 0, isz, ss->stream));
    CK(cudaMemsetAsync(ss->img2m, 0, isz, ss->stream));
    CK(cudaMemsetAsync(ss->illum, 0, isz, ss->stream));
    if (ss->o.extra_images)
        for (void *im : ss->ximg) CK(cudaMemsetAsync(im, 0, isz, ss->stream));
    CK(cudaStreamSynchronize(ss->stream));
    return RTM_OK;
}

void *rtm_session_stream(rtm_session *ss) { return ss ? (void *)ss->stream : nullptr; }

double rtm_session_kernel_ms(rtm_session *ss, const char *kernel, int *launches)
{
    if (launches) *launches = 0;
    if (!ss || !kernel) return -1;
    auto it = ss->timing.find(kernel);
    if (it == ss->timing.end() || it->second.used == 0) return -1;
    cudaStreamSynchronize(ss->stream);
    double tot = 0;
    for (int i = 0; i < it->second.used; i++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, it->second.ev[i].first, it->second.ev[i].second);
        tot += ms;
    }
    if (launches) *launches = it->second.used;
    return tot / it->second.used;
}

int rtm_session_get_wavefields(rtm_session *ss, int slot, float *ps, float *pr)
{
    if (!ss || slot < 0 || slot >= ss->last_batch_n) return fail(RTM_ERR_ARG, "bad slot");
    const ShotState &sh = ss->shots[ss->last_batch_shots[slot]];
    const Slot &sl = ss->slots[slot];
    CK(cudaSetDevice(ss->dev));
    if (ps) CK(cudaMemcpy2D(ps, sh.X * 4, sl.a.p, sh.pitch * 4, sh.X * 4, sh.Z, cudaMemcpyDeviceToHost));
    if (pr) CK(cudaMemcpy2D(pr, sh.X * 4, sl.b.p, sh.pitch * 4, sh.X * 4, sh.Z, cudaMemcpyDeviceToHost));
    return RTM_OK;
}

void rtm_session_close(rtm_session *ss)
{
    if (!ss) return;
    cudaSetDevice(ss->dev);
    if (ss->stream) cudaStreamSynchronize(ss->stream);
    for (auto &kv : ss->graphs) cudaGraphExecDestroy(kv.second.exec);
    ss->graphs.clear();
    for (auto &kv : ss->timing)
        for (auto &e : kv.second.ev) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    ss->interp.release();
    if (ss->arena.base) cudaFree(ss->arena.base);
    if (ss->stream) cudaStreamDestroy(ss->stream);
    delete ss;
}

int rtm_forward(const rtm_survey *s, const rtm_options *o, int ishot, const float *vp, const float *rho, int nsteps,
                float *p, float *vx, float *vz, float *gather)
{
    clear_error();
    if (!s || !o || !vp || !rho) return fail(RTM_ERR_ARG, "null argument");
    if (nsteps < 1 || nsteps > s->nt) return fail(RTM_ERR_ARG, "nsteps must be in [1, nt]");
    rtm_options oo = *o;
    oo.batch = 1;
    rtm_session *ss = nullptr;
    int rc = rtm_session_open(&ss, s, &oo, &ishot, 1, vp, rho, nullptr, nullptr, nullptr);
    if (rc) return rc;
    BatchRun br;
    const ShotState &sh = ss->shots[0];
    const Slot &sl = ss->slots[0];
    if (!(rc = batch_setup(ss, 0, 1, br)) && !(rc = batch_forward(ss, br, nsteps, false, true)) &&
        !(rc = settle_fields(ss, br))) {
        cudaError_t e = cudaStreamSynchronize(ss->stream);
        if (e != cudaSuccess) rc = fail(RTM_ERR_CUDA, cudaGetErrorString(e));
        if (!rc) rc = check_kernel_flag(ss);
        const size_t w = sizeof(float);
        if (!rc && p && cudaMemcpy2D(p, sh.X * w, sl.a.p, sh.pitch * w, sh.X * w, sh.Z, cudaMemcpyDeviceToHost))
            rc = fail(RTM_ERR_CUDA, "copy p");
        if (!rc && vx &&
            cudaMemcpy2D(vx, (sh.X - 1) * w, sl.a.vx, sh.pitch * w, (sh.X - 1) * w, sh.Z, cudaMemcpyDeviceToHost))
            rc = fail(RTM_ERR_CUDA, "copy vx");
        if (!rc && vz && cudaMemcpy2D(vz, sh.X * w, sl.a.vz, sh.pitch * w, sh.X * w, sh.Z - 1, cudaMemcpyDeviceToHost))
            rc = fail(RTM_ERR_CUDA, "copy vz");
        if (!rc && gather &&
            cudaMemcpy(gather, s->mode == 0 ? sh.gather_raw : sh.gather32, w * (size_t)nsteps * sh.g.nrec,
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(RTM_ERR_CUDA, "copy gather");
    }
    rtm_session_close(ss);
    return rc;
}

int rtm_migrate(const rtm_survey *s, const rtm_options *o, const int *shots, int nshots, const float *vp,
                const float *rho, const float *vp_mig, const float *rho_mig, const float *const *gathers_in,
                float *const *gathers_out, float *image1, float *image2s, float *image2m, float *illum,
                rtm_stats *stats)
{
    rtm_session *ss = nullptr;
    int rc = rtm_session_open(&ss, s, o, shots, nshots, vp, rho, vp_mig, rho_mig, nullptr);
    if (rc) return rc;
    if (s->mode == 1) {
        for (int k = 0; k < nshots; k++) {
            if (!gathers_in || !gathers_in[k]) {
                rtm_session_close(ss);
                return fail(RTM_ERR_ARG, "mode 1 needs a gather for every shot");
            }
            if ((rc = rtm_session_set_gather(ss, k, gathers_in[k]))) {
                rtm_session_close(ss);
                return rc;
            }
        }
    }
    if ((rc = rtm_session_run(ss, stats))) {
        rtm_session_close(ss);
        return rc;
    }
    if (s->mode == 0 && gathers_out)
        for (int k = 0; k < nshots; k++)
            if (gathers_out[k] && (rc = rtm_session_get_gather(ss, k, gathers_out[k]))) {
                rtm_session_close(ss);
                return rc;
            }
    rc = rtm_session_get_images(ss, image1, image2s, image2m, illum);
    rtm_session_close(ss);
    return rc;
}

int rtm_batch(const rtm_batch_desc *d, rtm_stats *stats)
{
    clear_error();
    if (!d) return fail(RTM_ERR_ARG, "null batch descriptor");
    return rtm_migrate(&d->survey, &d->options, d->shots, d->nshots, d->vp, d->rho, d->vp_mig, d->rho_mig,
                       d->gathers_in, d->gathers_out, d->image1, d->image2s, d->image2m, d->illum, stats);
}

}  // extern "C"
