// rtm_capi.cpp — extern "C" entry points: the drop-in rtm_model() and the host-side
// pieces of the path.  rtm_model keeps the reference's symbol, argument list and file side
// effects (gubingluo RTM_GPU_velstr.cpp:23-28, rtm_model.cu:12-17, :286-303, :490-538,
// :571-585) on top of the batched session engine.
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rtm_b200.h"
#include "rtm_internal.h"

namespace rtm {
int session_wave_size(const rtm_session *ss, int remaining);
int session_run_range(rtm_session *ss, int k0, int n);
}  // namespace rtm

using namespace rtm;

static int env_int(const char *name, int def)
{
    const char *v = std::getenv(name);
    return v && *v ? std::atoi(v) : def;
}
static int env_prec(const char *name)
{
    const char *v = std::getenv(name);
    if (!v) return RTM_PREC_FP32;
    if (!std::strcmp(v, "fp16")) return RTM_PREC_FP16;
    if (!std::strcmp(v, "bf16")) return RTM_PREC_BF16;
    return RTM_PREC_FP32;
}

// Runs the session's shots in batches and writes what the reference's drivers write: in mode
// 0 each modelled gather (rtm_model.cu:286-288), the ./output/ temp images after a batch
// holding a shot with (ishot-1)%50 == 0 (rtm_model.cu:490-538, rtm_real.cu:469-531; written
// with dx, as there), then the images (rtm_model.cu:575-585) and ./output/{idevice}Imagetrue.su.
static void drive(const char *who, rtm_session *ss, const rtm_survey &s, const rtm_options &o,
                  const std::vector<int> &shots, int idevice, int sgyflag, int endianflag, float *image1,
                  float *image2s, float *image3s, float *image4s, float *image5s, float *image2m, float *image3m,
                  float *image4m, float *image5m, float *illum)
{
    const int nx = s.nx, nz = s.nz, nt = s.nt, mode = s.mode;
    const float dx = s.dx;
    const size_t nimg = (size_t)nx * nz;
    char path[512];
    int rc;
    std::vector<float> tmp(nimg);
    std::vector<float> xi[7];   // image3s .. image5m, imagetrue (zero unless extra_images)
    for (auto &v : xi) v.assign(nimg, 0.0f);
    // checkpoint after every batch (RTM_B200_CHECKPOINT=<path>); resume from it
    // (RTM_B200_RESUME=1) when it exists and matches this run
    const char *ckpt = std::getenv("RTM_B200_CHECKPOINT");
    if (ckpt && !*ckpt) ckpt = nullptr;
    size_t start = 0;
    if (ckpt && env_int("RTM_B200_RESUME", 0)) {
        FILE *probe = std::fopen(ckpt, "rb");
        if (!probe) {
            std::printf("%s: no checkpoint at %s, starting from the first shot\n", who, ckpt);
        } else {
            std::fclose(probe);
            int done = 0;
            if (rtm_session_load_checkpoint(ss, ckpt, &done)) {
                std::printf("%s: %s\n", who, rtm_last_error());
                return;
            }
            start = (size_t)done;
            std::printf("%s: resuming after %d of %zu shots from %s\n", who, done, shots.size(), ckpt);
        }
    }
    // one JSON line per batch (RTM_B200_LOG=<path>)
    FILE *log = nullptr;
    if (const char *lp = std::getenv("RTM_B200_LOG"))
        if (*lp) log = std::fopen(lp, "a");
    for (size_t k0 = start; k0 < shots.size();) {
        const int n = session_wave_size(ss, (int)(shots.size() - k0));
        auto t0 = std::chrono::steady_clock::now();
        rc = session_run_range(ss, (int)k0, n);
        if (rc) {
            std::printf("%s: %s\n", who, rtm_last_error());
            if (log) std::fclose(log);
            return;   // the caller closes the session
        }
        double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (ckpt && rtm_session_save_checkpoint(ss, ckpt, (int)(k0 + n)))
            std::printf("%s: %s\n", who, rtm_last_error());
        if (log) {
            std::fprintf(log, "{\"entry\": \"%s\", \"first_shot\": %d, \"last_shot\": %d, \"shots\": %d, "
                              "\"seconds\": %.6f, \"shots_per_s\": %.6f, \"shots_done\": %zu, \"shots_total\": %zu}\n",
                         who, shots[k0], shots[k0 + n - 1], n, sec, n / sec, k0 + n, shots.size());
            std::fflush(log);
        }
        bool temp_dump = false;
        for (int j = 0; j < n; j++) {
            const int ishot = shots[k0 + j];
            if (mode == 0) {   // rtm_model.cu:286-288
                rtm_geometry g;
                shot_geometry(s, ishot, g);
                std::vector<float> gat((size_t)nt * g.nrec);
                rtm_session_get_gather(ss, (int)(k0 + j), gat.data());
                std::snprintf(path, sizeof(path), "./seisReal/%dseisreal.su", ishot);
                if (write_gather_su(path, gat.data(), g, nt, sgyflag, endianflag))
                    std::printf("The file %s open failed !\n", path);
            }
            if ((ishot - 1) % 50 == 0) temp_dump = true;
            std::printf("%d shot finished: %g (s)\n", ishot, sec / n);
        }
        if (temp_dump) {   // rtm_model.cu:490-538 (images are written with dx, as there)
            float *outs[4] = {image1, image2s, image2m, illum};
            rtm_session_get_images(ss, outs[0] ? outs[0] : tmp.data(), image2s ? image2s : tmp.data(),
                                   image2m ? image2m : tmp.data(), illum ? illum : tmp.data());
            if (o.extra_images)
                rtm_session_get_images_extra(ss, xi[0].data(), xi[1].data(), xi[2].data(), xi[3].data(),
                                             xi[4].data(), xi[5].data(), xi[6].data());
            struct {
                const char *name;
                const float *img;
            } temps[] = {{"Image2stemp", image2s}, {"Image3stemp", xi[0].data()}, {"Image4stemp", xi[1].data()},
                         {"Image5stemp", xi[2].data()}, {"Image1temp", image1}, {"Illumtemp", illum},
                         {"Image2mtemp", image2m}, {"Image3mtemp", xi[3].data()}, {"Image4mtemp", xi[4].data()},
                         {"Image5mtemp", xi[5].data()}, {"Imagetruetemp", xi[6].data()}};
            for (auto &t : temps) {
                if (!t.img) continue;
                std::snprintf(path, sizeof(path), "./output/%s.su", t.name);
                if (write_image_su(path, t.img, nz, nx, dx)) std::printf("The file %s open failed !\n", path);
            }
        }
        k0 += n;
    }
    if (log) std::fclose(log);
    rtm_session_get_images(ss, image1, image2s, image2m, illum);   // rtm_model.cu:575-585
    if (o.extra_images)
        rtm_session_get_images_extra(ss, image3s, image4s, image5s, image3m, image4m, image5m, xi[6].data());
    std::snprintf(path, sizeof(path), "./output/%dImagetrue.su", idevice);
    if (write_image_su(path, xi[6].data(), nz, nx, dx)) std::printf("The file %s open failed !\n", path);
}

extern "C" {

void rtm_model(int idevice, int nshot, int startshot, int dshot, int mode, int medium_flag, int flag_layout,
               int sgyflag, int endianflag, int ismth, int nx, int nz, int nt, float dx, float dz, float dt, int npml,
               float direct, float direct0, float tsnap, float fdom, float spx0, float spz0, float dspx, float offset,
               float offsetmax, float amp, float alp, float *vp0, float *rho0, float *diffcoef, float *wavelet,
               float *image1, float *image2s, float *image3s, float *image4s, float *image5s, float *image2m,
               float *image3m, float *image4m, float *image5m, float *illum)
{
    (void)wavelet;   // the reference regenerates the wavelet on the device (rtm_model.cu:86-88)
    clear_error();
    rtm_survey s;
    std::memset(&s, 0, sizeof(s));
    s.nx = nx; s.nz = nz; s.nt = nt; s.dx = dx; s.dz = dz; s.dt = dt; s.npml = npml;
    s.fdom = fdom; s.amp = amp; s.alp = alp; s.layout = flag_layout;
    s.spx0 = spx0; s.spz0 = spz0; s.dspx = dspx; s.offset = offset; s.offsetmax = offsetmax;
    s.mode = mode; s.medium_flag = medium_flag; s.ismth = ismth;
    s.direct = direct; s.direct0 = direct0; s.mute = 1;
    s.receiver_depth = env_int("RTM_B200_RECEIVER_DEPTH", 0);
    rtm_options o;
    std::memset(&o, 0, sizeof(o));
    o.device = idevice;
    o.strip_precision = env_prec("RTM_B200_STRIPS");
    o.gather_precision = env_prec("RTM_B200_GATHERS");
    o.accum_fp64 = env_int("RTM_B200_ACCUM_FP64", 0);
    o.batch = env_int("RTM_B200_BATCH", 0);
    o.verbose = 1;
    o.tsnap = tsnap;
    // image3*/4*/5* and Imagetrue: the reference's other imaging conditions, with vx and vz
    // read at their own cells (1, the default) or with the reference's indexing (2); 0 leaves
    // those images zero and saves their cost
    o.extra_images = env_int("RTM_B200_EXTRA_IMAGES", 1);
    const size_t nimg = (size_t)nx * nz;
    float *zero_imgs[6] = {image3s, image4s, image5s, image3m, image4m, image5m};
    for (float *p : zero_imgs)
        if (p) std::memset(p, 0, nimg * sizeof(float));

    std::vector<int> shots;
    for (int ishot = startshot; ishot <= nshot; ishot += (dshot > 0 ? dshot : 1)) shots.push_back(ishot);
    if (shots.empty()) {
        std::printf("rtm_model: no shots between %d and %d\n", startshot, nshot);
        return;
    }
    rtm_session *ss = nullptr;
    int rc = rtm_session_open(&ss, &s, &o, shots.data(), (int)shots.size(), vp0, rho0, nullptr, nullptr, diffcoef);
    if (rc) {
        std::printf("rtm_model: %s\n", rtm_last_error());
        return;
    }
    char path[512];
    if (mode == 1) {
        for (size_t k = 0; k < shots.size(); k++) {
            std::snprintf(path, sizeof(path), "./seisReal/%dseisreal.su", shots[k]);
            int nt_f = 0, ntr_f = 0;
            rc = read_gather_su(path, sgyflag, nullptr, &nt_f, &ntr_f, nullptr);
            if (!rc && (nt_f != nt || ntr_f != rtm_session_nrec(ss, (int)k)))
                rc = fail(RTM_ERR_IO, std::string(path) + " does not match nt/receiver count of the shot");
            std::vector<float> g;
            if (!rc) {
                g.resize((size_t)nt_f * ntr_f);
                rc = read_gather_su(path, sgyflag, g.data(), nullptr, nullptr, nullptr);
            }
            if (!rc) rc = rtm_session_set_gather(ss, (int)k, g.data());
            if (rc) {
                std::printf("rtm_model: %s\n", rtm_last_error());
                rtm_session_close(ss);
                return;
            }
        }
    }
    drive("rtm_model", ss, s, o, shots, idevice, sgyflag, endianflag, image1, image2s, image3s, image4s, image5s,
          image2m, image3m, image4m, image5m, illum);
    rtm_session_close(ss);
}

void rtm_real(int idevice, int nshot, int startshot, int dshot, int medium_flag, int flag_layout, int sgyflag,
              int endianflag, int ismth, int nx, int nz, int nt, float dx, float dz, float dt, int nx0, int nz0, int nt0,
              float dx0, float dz0, float dt0, int npml, int lx, int lz, float tsnap, float fdom, float spz0, float amp,
              float alp, float direct, float direct0, float *vp0, float *rho0, float *diffcoef, float *wavelet,
              char filename_shotgather[40], int **shotprofileId, float *image1, float *image2s, float *image3s,
              float *image4s, float *image5s, float *image2m, float *image3m, float *image4m, float *image5m,
              float *illum)
{
    // accepted and unused, as in the reference (rtm_real.cu:17-581)
    (void)flag_layout; (void)nx0; (void)nz0; (void)dz0; (void)lx; (void)lz; (void)wavelet;
    clear_error();
    rtm_survey s;
    std::memset(&s, 0, sizeof(s));
    s.nx = nx; s.nz = nz; s.nt = nt; s.dx = dx; s.dz = dz; s.dt = dt; s.npml = npml;
    s.fdom = fdom; s.amp = amp; s.alp = alp; s.layout = 3; s.spz0 = spz0;
    s.mode = 1; s.medium_flag = medium_flag; s.ismth = ismth;
    s.direct = direct; s.direct0 = direct0;
    s.mute = 2;   // rtm_real.cu:397-403: the mute reads the velocities after smoothing
    s.receiver_depth = env_int("RTM_B200_RECEIVER_DEPTH", 0);
    rtm_options o;
    std::memset(&o, 0, sizeof(o));
    o.device = idevice;
    o.strip_precision = env_prec("RTM_B200_STRIPS");
    o.gather_precision = env_prec("RTM_B200_GATHERS");
    o.accum_fp64 = env_int("RTM_B200_ACCUM_FP64", 0);
    o.batch = env_int("RTM_B200_BATCH", 0);
    o.verbose = 1;
    o.extra_images = env_int("RTM_B200_EXTRA_IMAGES", 1);
    o.tsnap = tsnap;
    const int mirror = env_int("RTM_B200_FK_MIRROR", 0);
    const size_t nimg = (size_t)nx * nz;
    float *zero_imgs[6] = {image3s, image4s, image5s, image3m, image4m, image5m};
    for (float *p : zero_imgs)
        if (p) std::memset(p, 0, nimg * sizeof(float));
    if (!shotprofileId || !filename_shotgather) {
        fail(RTM_ERR_ARG, "null shot table or file name");
        std::printf("rtm_real: %s\n", rtm_last_error());
        return;
    }
    std::vector<int> shots;
    for (int ishot = startshot; ishot <= nshot; ishot += (dshot > 0 ? dshot : 1)) shots.push_back(ishot);
    if (shots.empty()) {
        std::printf("rtm_real: no shots between %d and %d\n", startshot, nshot);
        return;
    }
    // per-shot geometry from the scanned table (rtm_real.cu:134-157)
    std::vector<rtm_geometry> geoms(shots.size());
    std::vector<int> ncols0(shots.size());
    for (size_t k = 0; k < shots.size(); k++) {
        const int i = shots[k] - 1;
        if (i < 0) {
            std::printf("rtm_real: shot numbers start at 1\n");
            return;
        }
        int rc = real_geometry(s, shotprofileId[0][i], shotprofileId[3][i], shotprofileId[1][i], dx0, geoms[k],
                               &ncols0[k]);
        if (rc) {
            std::printf("rtm_real: shot %d: %s\n", shots[k], rtm_last_error());
            return;
        }
        geoms[k].iTraceAll = shotprofileId[2][i];
    }
    rtm_session *ss = nullptr;
    int rc = rtm_session_open_geometry(&ss, &s, &o, shots.data(), geoms.data(), (int)shots.size(), vp0, rho0,
                                       nullptr, nullptr, diffcoef);
    if (rc) {
        std::printf("rtm_real: %s\n", rtm_last_error());
        return;
    }
    // recorded traces (rtm_real.cu:379-394), resampled and muted on the device (:395-403)
    char path[512];
    std::snprintf(path, sizeof(path), "./seisReal/%s", filename_shotgather);
    std::vector<float> obs;
    for (size_t k = 0; k < shots.size() && !rc; k++) {
        const int i = shots[k] - 1;
        obs.assign((size_t)nt0 * ncols0[k], 0.0f);
        rc = read_shot_traces(path, sgyflag, endianflag, nt0, shotprofileId[2][i], shotprofileId[1][i], ncols0[k],
                              obs.data());
        if (!rc) rc = rtm_session_set_gather_raw(ss, (int)k, obs.data(), ncols0[k], nt0, dt0, mirror);
        if (rc) std::printf("rtm_real: shot %d: %s\n", shots[k], rtm_last_error());
    }
    if (!rc)
        drive("rtm_real", ss, s, o, shots, idevice, sgyflag, endianflag, image1, image2s, image3s, image4s, image5s,
              image2m, image3m, image4m, image5m, illum);
    rtm_session_close(ss);
}

int rtm_scan_shotgather(const char *path, int sgyflag, int *endianflag, int *profile, int max_shots)
{
    clear_error();
    int n = 0;
    int rc = scan_shotgather(path, sgyflag, endianflag, profile, max_shots, &n);
    return rc ? rc : n;
}

int rtm_real_geometry(const rtm_survey *s, int sx, int offset, int ntrace, float dx0, rtm_geometry *g, int *ncols0)
{
    clear_error();
    if (!s || !g) return fail(RTM_ERR_ARG, "null argument");
    return real_geometry(*s, sx, offset, ntrace, dx0, *g, ncols0);
}

int rtm_read_shot_traces(const char *path, int sgyflag, int endianflag, int nt0, long long itrace_all, int ntrace,
                         int ncols, float *seisobs)
{
    clear_error();
    return read_shot_traces(path, sgyflag, endianflag, nt0, itrace_all, ntrace, ncols, seisobs);
}

int rtm_shot_geometry(const rtm_survey *s, int ishot, rtm_geometry *g)
{
    if (!s || !g) return fail(RTM_ERR_ARG, "null argument");
    return shot_geometry(*s, ishot, *g);
}

void rtm_coef_table(float *c100) { coef_table(c100); }

int rtm_prepare_model(const float *vp, const float *rho, int nx, int nz, int nx1, int nx2, int npml, int medium_flag,
                      float *vp2_pad, float *rho_pad)
{
    if (!vp || nx1 < 0 || nx2 >= nx || nx2 < nx1 || npml < 0) return fail(RTM_ERR_ARG, "bad model window");
    const int X = nx2 - nx1 + 1 + 2 * npml, Z = nz + 2 * npml;
    if (vp2_pad) {
        extract_extend(vp, nx, nz, nx1, nx2, npml, true, vp2_pad);
        if (medium_flag) pml_smooth(vp2_pad, X, Z, npml);
    }
    if (rho && rho_pad) {
        extract_extend(rho, nx, nz, nx1, nx2, npml, false, rho_pad);
        if (medium_flag) pml_smooth(rho_pad, X, Z, npml);
    }
    return RTM_OK;
}

int rtm_velsmooth(float *a, int n1, int n2, int nsp)
{
    if (!a || n1 < 1 || n2 < 1 || nsp < 0) return fail(RTM_ERR_ARG, "bad smoothing argument");
    gauss_smooth(a, n1, n2, nsp);
    return RTM_OK;
}

int rtm_pmlsmooth(float *a, int nxpad, int nzpad, int npml)
{
    if (!a || nxpad < 3 || nzpad < 3 || npml < 1) return fail(RTM_ERR_ARG, "bad smoothing argument");
    pml_smooth(a, nxpad, nzpad, npml);
    return RTM_OK;
}

int rtm_interp_model(const float *vp0, float *vp, int nx0, int nz0, int nx, int nz, int lx, int lz)
{
    if (!vp0 || !vp || lx < 1 || lz < 1 || nx != (nx0 - 1) * lx + 1 || nz != (nz0 - 1) * lz + 1)
        return fail(RTM_ERR_ARG, "bad interpolation sizes");
    interp_model(vp0, vp, nx0, nz0, nx, lx, lz);
    return RTM_OK;
}

void rtm_get_constant(const float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0, float dt0,
                      float *dx, float *dz, int *nx, int *nz, int *nt, float *dt, int *lx, int *lz, float *vpmin,
                      float *vpmax)
{
    get_constant(vp, fdom, dx0, dz0, nx0, nz0, nt0, dt0, dx, dz, nx, nz, nt, dt, lx, lz, vpmin, vpmax);
}

void rtm_laplace_image(float *image, int nx, int nz, int dx, int dz) { laplace_image(image, nx, nz, dx, dz); }
void rtm_scale_image(const float *illum, float *image, int n) { scale_image(illum, image, n); }

int rtm_read_params(const char *input_dir, rtm_params *p)
{
    if (!p) return fail(RTM_ERR_ARG, "null argument");
    return read_params(input_dir, *p);
}
int rtm_read_velocity(const char *path, int nx, int nz, float *vp)
{
    if (!path || !vp || nx < 1 || nz < 1) return fail(RTM_ERR_ARG, "bad argument");
    return read_velocity(path, nx, nz, vp);
}
int rtm_write_image_su(const char *path, const float *image, int nz, int nx, float d)
{
    if (!path || !image) return fail(RTM_ERR_ARG, "bad argument");
    return write_image_su(path, image, nz, nx, d);
}
int rtm_write_gather_su(const char *path, const float *gather, const rtm_geometry *g, int nt, int sgyflag,
                        int endianflag)
{
    if (!path || !gather || !g) return fail(RTM_ERR_ARG, "bad argument");
    return write_gather_su(path, gather, *g, nt, sgyflag, endianflag);
}
int rtm_read_gather_su(const char *path, int sgyflag, float *gather, int *nt, int *ntr, rtm_geometry *keys)
{
    if (!path) return fail(RTM_ERR_ARG, "bad argument");
    return read_gather_su(path, sgyflag, gather, nt, ntr, keys);
}

}  // extern "C"
