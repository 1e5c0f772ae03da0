// rtm_internal.h — declarations shared by the library's translation units.
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "rtm_b200.h"

struct CUstream_st;
typedef CUstream_st *cudaStream_t_fwd;   // cudaStream_t without the runtime header

namespace rtm {

int fail(int code, const std::string &msg);
void clear_error();
const char *last_error();

void coef_table(float *c100);
int shot_geometry(const rtm_survey &s, int ishot, rtm_geometry &g);
void extract_extend(const float *v, int nx, int nz, int nx1, int nx2, int npml, bool square, float *pad);
void pml_smooth(float *vp, int nx, int nz, int npml);
void gauss_smooth(float *vp, int n1, int n2, int nsp);
void interp_model(const float *vp0, float *vp, int nx0, int nz0, int nx, int lx, int lz);
void get_constant(const float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0, float dt0,
                  float *dx, float *dz, int *nx, int *nz, int *nt, float *dt, int *lx, int *lz, float *vpmin,
                  float *vpmax);
void laplace_image(float *image, int nx, int nz, int dx, int dz);
void scale_image(const float *illum, float *grad, int n);

int read_velocity(const char *path, int nx, int nz, float *vp);
int write_image_su(const char *path, const float *image, int nz, int nx, float d);
int write_gather_su(const char *path, const float *gather, const rtm_geometry &g, int nt, int sgyflag,
                    int endianflag);
int read_gather_su(const char *path, int sgyflag, float *gather, int *nt, int *ntr, rtm_geometry *keys);
int read_params(const char *input_dir, rtm_params &p);

// ---- real-data path --------------------------------------------------------------------
int scan_shotgather(const char *path, int sgyflag, int *endianflag, int *profile, int max_shots, int *nshots);
int real_geometry(const rtm_survey &s, int sx, int offset, int ntrace, float dx0, rtm_geometry &g, int *ncols0);
int read_shot_traces(const char *path, int sgyflag, int endianflag, int nt0, long long itrace_all, int ntrace,
                     int ncols, float *seisobs);

// Shape of one gather interpolation [nt0][nx0] -> [nt][nx] (reference Interpseis2d).
struct InterpShape {
    int nx0, nt0, nx, nt;
    int fk, sinc;          // x by F-K (nx > nx0), t by sinc (nt > nt0)
    int lx, Nx, Nt, nf;    // F-K: fold, padded sizes, positive frequencies
};
int interp_shape(int nx0, int nt0, int nx, int nt, InterpShape &sh);

// Device workspace and cuFFT plans of one shape; kept by the caller and reused while the
// shape repeats (shots of a survey usually share it).
struct InterpPlan {
    InterpShape shape{};
    void *work = nullptr;                 // one allocation holding everything below
    float *d_in = nullptr, *d_tmp = nullptr;
    void *K = nullptr, *S = nullptr, *Z = nullptr, *G1 = nullptr, *G = nullptr;   // double2 arrays
    unsigned *zmax = nullptr;
    int p_k = 0, p_s = 0, p_x = 0, p_t = 0;   // cufftHandle values, valid when `plans`
    bool plans = false;
    std::vector<std::pair<size_t, size_t>> guards;   // checking mode: (offset, length) bands
    void release();
};
// Checking mode (RTM_B200_GUARDS=1): the guard bands after the workspace's buffers are intact.
int interp_check_guards(const InterpPlan &p);
// Uploads host_in [nt0][nx0] and writes the interpolated gather to d_out [nt][nx] on stream
// st; mirror 0 = the reference's negative-frequency indexing, 1 = the Hermitian partner.
int interp_gather_device(InterpPlan &p, const float *host_in, int nx0, int nt0, float *d_out, int nx, int nt,
                         float dt, float dt0, int mirror, cudaStream_t_fwd st, int *launches);

}  // namespace rtm
