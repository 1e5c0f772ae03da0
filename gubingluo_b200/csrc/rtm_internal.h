// rtm_internal.h — declarations shared by the library's translation units.
#pragma once
#include <string>

#include "rtm_b200.h"

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

}  // namespace rtm
