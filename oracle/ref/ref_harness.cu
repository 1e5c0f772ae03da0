// ref_harness.cu — runs the reference's own CUDA code (rebuilt from its sources for sm_100a)
// to produce golden vectors for the oracle.  TEST INFRASTRUCTURE ONLY.
//
// The reference's kernels and shot driver are compiled as one translation unit (its
// kernel.cu, then its rtm_model.cu); an empty kernel.cuh stands in for the header the
// reference does not ship.  Every device allocation the reference makes is padded by 1 MiB:
// its bottom-edge pressure-PML kernels read one row past the end of vz and one element
// past the end of vx (kernel.cu:905, :1123), and the padding keeps those reads inside the
// allocation.  All grids used here have nxlen, nz, nxpad and nzpad multiples of 32, the
// sizes for which every reference guard around __syncthreads is uniform across a block.
//
//   ref_harness units <dir>      unit kernels + 300 forward / 20 backward steps
//   ref_harness rtm <dir>        three rtm_model() runs (layouts 1 and 2, modes 0 and 1)
//   ref_harness time <dir> <case> per-shot timing of rtm_model() at a larger parity size
//   ref_harness real <dir>       scanshotgather() + rtm_real() on a synthetic 3-shot SEG-Y
//                                file (called with rtm_real.cu's own argument list)
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static cudaError_t harness_malloc(void **p, size_t n) { return cudaMalloc(p, n + ((size_t)1 << 20)); }

#include "kernel.cu"
#define cudaMalloc(ptr, n) harness_malloc((void **)(ptr), (n))
#include "rtm_model.cu"
#include "rtm_real.cu"
#undef cudaMalloc

// scanshotgather is defined in the reference's RTM_GPU_velstr.cpp (compiled with its main
// renamed).
void scanshotgather(char filename_shotgather[40], int **shotprofileId, int sgyflag, int *endianflag);

static std::string g_dir;

static void ck(const char *what)
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error after %s: %s\n", what, cudaGetErrorString(e));
        std::exit(2);
    }
}

template <typename T>
static void dump_host(const char *name, const T *h, size_t n)
{
    std::string path = g_dir + "/" + name + (sizeof(T) == 4 && (T)0.5 == 0 ? ".i32" : ".f32");
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(3); }
    std::fwrite(h, sizeof(T), n, f);
    std::fclose(f);
}

template <typename T>
static void dump_dev(const char *name, const T *d, size_t n)
{
    std::vector<T> h(n);
    cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    ck(name);
    dump_host(name, h.data(), n);
}

template <typename T>
static T *dalloc(size_t n)
{
    T *p = nullptr;
    harness_malloc((void **)&p, n * sizeof(T));
    cudaMemset(p, 0, n * sizeof(T) + ((size_t)1 << 20));
    return p;
}

static void coef_table(float *diffcoef)
{
    // RTM_GPU_velstr.cpp:184-196
    std::memset(diffcoef, 0, 100 * sizeof(float));
    for (int ix = 0; ix < 10; ix++) {
        int N1 = 2 * (ix + 1);
        float tmp[10];
        Diff_coeffVelStrLiuyang(tmp, N1);
        for (int iz = 0; iz < N1 / 2; iz++) diffcoef[ix * 10 + iz] = tmp[iz];
    }
}

// Smooth heterogeneous model used by the golden runs (velocity in m/s, density in kg/m^3).
static void make_model(int nx, int nz, float dx, float *vp, float *rho, int variant)
{
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
            float z = iz * dx, x = ix * dx;
            float v = 2000.0f + 1.2f * z;
            if (z > 380.0f + 0.15f * x) v += 700.0f;              // dipping interface
            float bx = x - 0.55f * nx * dx, bz = z - 0.45f * nz * dx;
            if (bx * bx + bz * bz < 90.0f * 90.0f) v -= 400.0f;   // slow lens
            if (variant) v += 60.0f * sinf(0.031f * x) * cosf(0.047f * z);
            vp[iz * nx + ix] = v;
            rho[iz * nx + ix] = variant ? 1800.0f + 0.25f * v : 2000.0f;
        }
}

static void mkdir_p(const std::string &d) { mkdir(d.c_str(), 0755); }

// ---------------------------------------------------------------------------------------
static int run_units()
{
    const int nxl = 96, nzl = 64, npml = 32, X = nxl + 2 * npml, Z = nzl + 2 * npml;
    const float dx = 10.0f, dz = 10.0f, dt = 1.0e-3f, fdom = 25.0f;
    const int nt = 400, nsx = 70, nsz = 34, nsteps = 300, nback = 20;
    const float amp = 1.0f, alp = 0.07f, vpmax_prof = 3000.0f;
    const float dx2 = dx * dx, dz2 = dz * dz, _dtx = dt / dx, _dtz = dt / dz;
    float _dt = 1.0 / dt;
    dim3 blk(Block_Sizez, Block_Sizex);
    dim3 gfull((Z + 31) / 32, (X + 31) / 32);
    dim3 gp((Z - 2 * npml + 31) / 32, (X - 2 * npml + 31) / 32);
    dim3 gvx((Z + 31) / 32, (X - 2 * npml - 1 + 31) / 32);
    dim3 gvz((Z - 2 * npml - 1 + 31) / 32, (X + 31) / 32);
    dim3 gvxb((Z - 2 * npml + 31) / 32, (X - 2 * npml - 1 + 31) / 32);
    dim3 gvzb((Z - 2 * npml - 1 + 31) / 32, (X - 2 * npml + 31) / 32);
    dim3 gvxlr((Z + 31) / 32, 2), gvztb(2, (X + 31) / 32);
    dim3 gplr((Z - 2 * npml + 31) / 32, 2), gptb(2, (X - 2 * npml + 31) / 32), gcor(2, 2);
    dim3 grec((nt + 31) / 32, (X - 2 * npml + 31) / 32);
    dim3 bpmllr(Block_Sizez, 10), bpmltb(10, Block_Sizex);
    dim3 gpmllr((Z - 2 * npml + 31) / 32, 2), gpmltb(2, (X - 2 * npml + 31) / 32);

    float *d_ddx = dalloc<float>(X), *d_ddz = dalloc<float>(Z);
    float *d_ddxVx = dalloc<float>(X - 1), *d_ddzVz = dalloc<float>(Z - 1);
    cuda_pmlCoeffpx<<<(X + 127) / 128, 128>>>(d_ddx, vpmax_prof, dx, npml, X);
    cuda_pmlCoeffpz<<<(Z + 127) / 128, 128>>>(d_ddz, vpmax_prof, dz, npml, Z);
    cuda_pmlCoeffvx<<<(X + 126) / 128, 128>>>(d_ddxVx, vpmax_prof, dx, npml, X - 1);
    cuda_pmlCoeffvz<<<(Z + 126) / 128, 128>>>(d_ddzVz, vpmax_prof, dz, npml, Z - 1);
    ck("pml profiles");
    dump_dev("pml_ddx", d_ddx, X);
    dump_dev("pml_ddz", d_ddz, Z);
    dump_dev("pml_ddxvx", d_ddxVx, X - 1);
    dump_dev("pml_ddzvz", d_ddzVz, Z - 1);

    int *d_norder = dalloc<int>((size_t)X * Z), *d_norderx = dalloc<int>(X - 1), *d_norderz = dalloc<int>(Z - 1);
    cuda_norder<<<gfull, blk>>>(d_norder, X, Z);
    cuda_norderx<<<(X + 126) / 128, 128>>>(d_norderx, X - 1);
    cuda_norderz<<<(Z + 126) / 128, 128>>>(d_norderz, Z - 1);
    ck("norder");
    dump_dev("norder", d_norder, (size_t)X * Z);
    dump_dev("norderx", d_norderx, X - 1);
    dump_dev("norderz", d_norderz, Z - 1);

    float *d_w = dalloc<float>(nt);
    cuda_ricker_wavelet<<<(nt + 511) / 512, 512>>>(d_w, fdom, dt, nt);
    ck("ricker");
    dump_dev("ricker", d_w, nt);

    float *d_src = dalloc<float>((size_t)X * Z);
    cuda_source<<<gfull, blk>>>(d_src, nsx, nsz, X, Z, amp, alp, dx2, dz2);
    ck("source");
    dump_dev("source", d_src, (size_t)X * Z);

    // model (padded the way the reference's rtm_model pads it: extract + square + edge replicate)
    std::vector<float> v(nxl * nzl), r(nxl * nzl), vp2(X * Z), rho(X * Z), tmp(nxl * nzl);
    make_model(nxl, nzl, dx, v.data(), r.data(), 1);
    dump_host("model_v", v.data(), v.size());
    dump_host("model_rho", r.data(), r.size());
    extractvel1(tmp.data(), v.data(), nxl, nzl, 0, nxl - 1);
    extendvel1(vp2.data(), tmp.data(), nxl, nzl, npml);
    extractrho1(tmp.data(), r.data(), nxl, nzl, 0, nxl - 1);
    extendvel1(rho.data(), tmp.data(), nxl, nzl, npml);
    float vpmax = sqrtf(Maxval1(vp2.data(), X * Z));
    float *d_vp = dalloc<float>((size_t)X * Z), *d_rho = dalloc<float>((size_t)X * Z);
    cudaMemcpy(d_vp, vp2.data(), sizeof(float) * X * Z, cudaMemcpyHostToDevice);
    cudaMemcpy(d_rho, rho.data(), sizeof(float) * X * Z, cudaMemcpyHostToDevice);

    // mute of an all-ones gather (rtm_model.cu:289 launch shape)
    {
        int nw = (int)(1.5f / (fdom * dt)), tlength = (int)(0.05f / dt);
        std::vector<float> ones((size_t)nt * nxl, 1.0f);
        float *d_rec = dalloc<float>((size_t)nt * nxl);
        cudaMemcpy(d_rec, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice);
        cuda_mute1<<<grec, blk>>>(d_rec, d_vp, nsx, nsz, nt, npml, nxl, nw, tlength, fdom, dx2, dz2, _dt);
        ck("mute");
        dump_dev("mute_mask", d_rec, (size_t)nt * nxl);
        int meta[2] = {nw, tlength};
        dump_host("mute_meta", meta, 2);
    }
    // taper (rtm_model.cu:462-466)
    {
        int nwin = 50;
        while (2 * nwin >= nxl) nwin -= 3;
        float *d_taper = dalloc<float>((size_t)nxl * nzl);
        cuda_taper_calculate<<<gp, blk>>>(d_taper, nxl, nzl, nwin, 0.06f);
        ck("taper");
        dump_dev("taper", d_taper, (size_t)nxl * nzl);
    }

    // PML profiles of the model actually used for the steps below
    cudaMemset(d_ddx, 0, X * 4); cudaMemset(d_ddz, 0, Z * 4);
    cudaMemset(d_ddxVx, 0, (X - 1) * 4); cudaMemset(d_ddzVz, 0, (Z - 1) * 4);
    cuda_pmlCoeffpx<<<(X + 127) / 128, 128>>>(d_ddx, vpmax, dx, npml, X);
    cuda_pmlCoeffpz<<<(Z + 127) / 128, 128>>>(d_ddz, vpmax, dz, npml, Z);
    cuda_pmlCoeffvx<<<(X + 126) / 128, 128>>>(d_ddxVx, vpmax, dx, npml, X - 1);
    cuda_pmlCoeffvz<<<(Z + 126) / 128, 128>>>(d_ddzVz, vpmax, dz, npml, Z - 1);
    float coef[100];
    coef_table(coef);
    float *d_coef = dalloc<float>(100);
    cudaMemcpy(d_coef, coef, sizeof(coef), cudaMemcpyHostToDevice);

    float *d_p = dalloc<float>((size_t)X * Z), *d_vx = dalloc<float>((size_t)(X - 1) * Z), *d_vz = dalloc<float>((size_t)X * (Z - 1));
    float *d_pl1 = dalloc<float>(npml * Z), *d_pl2 = dalloc<float>(npml * Z), *d_pr1 = dalloc<float>(npml * Z), *d_pr2 = dalloc<float>(npml * Z);
    float *d_pt1 = dalloc<float>(npml * nxl), *d_pt2 = dalloc<float>(npml * nxl), *d_pb1 = dalloc<float>(npml * nxl), *d_pb2 = dalloc<float>(npml * nxl);
    float *d_gather = dalloc<float>((size_t)nsteps * nxl);
    const size_t lv = (size_t)20 * nzl, lh = (size_t)20 * nxl;
    float *d_svx = dalloc<float>(lv * nsteps), *d_svz = dalloc<float>(lh * nsteps);
    float *d_splr = dalloc<float>(lv * nsteps), *d_sptb = dalloc<float>(lh * nsteps);
    for (int it = 0; it < nsteps; it++) {   // rtm_model.cu:326-345, strips kept on the device
        cuda_forward_vx<<<gvx, blk>>>(d_p, d_vx, d_rho, d_coef, _dtx, npml, X, Z);
        cuda_forward_vz<<<gvz, blk>>>(d_p, d_vz, d_rho, d_coef, _dtz, npml, X, Z);
        cuda_pml_vxlr<<<gvxlr, blk>>>(d_p, d_vx, d_rho, d_coef, d_ddxVx, _dtx, dt, npml, X, Z, d_norderx);
        cuda_pml_vztb<<<gvztb, blk>>>(d_p, d_vz, d_rho, d_coef, d_ddzVz, _dtz, dt, npml, X, Z, d_norderz);
        cuda_forward_p<<<gp, blk>>>(d_p, d_vx, d_vz, d_rho, d_vp, d_coef, _dtx, _dtz, npml, X, Z);
        cuda_pml_plr<<<gplr, blk>>>(d_p, d_vx, d_vz, d_pl1, d_pl2, d_pr1, d_pr2, d_rho, d_vp, d_coef, d_ddx, d_ddz, _dtx, _dtz, dt, npml, X, Z, d_norder);
        cuda_pml_ptb<<<gptb, blk>>>(d_p, d_vx, d_vz, d_pt1, d_pt2, d_pb1, d_pb2, d_rho, d_vp, d_coef, d_ddz, _dtx, _dtz, dt, npml, X, Z, d_norder);
        cuda_pml_pconner<<<gcor, blk>>>(d_p, d_vx, d_vz, d_pl1, d_pl2, d_pr1, d_pr2, d_rho, d_vp, d_coef, d_ddx, d_ddz, _dtx, _dtz, dt, npml, X, Z, d_norder);
        cuda_add_source<<<gfull, blk>>>(d_p, d_src, d_w, dt, 1, X, Z, it);
        cuda_record1<<<(nxl + 127) / 128, 128>>>(d_p, &d_gather[(size_t)it * nxl], npml, nxl);
        save_d_vxpml<<<gpmllr, bpmllr>>>(d_vx, d_svx + lv * it, X, Z, npml);
        save_d_vzpml<<<gpmltb, bpmltb>>>(d_vz, d_svz + lh * it, X, Z, npml);
        save_d_ppmllr<<<gpmllr, bpmllr>>>(d_p, d_splr + lv * it, X, Z, npml);
        save_d_ppmltb<<<gpmltb, bpmltb>>>(d_p, d_sptb + lh * it, X, Z, npml);
    }
    ck("forward steps");
    dump_dev("fwd_p", d_p, (size_t)X * Z);
    dump_dev("fwd_vx", d_vx, (size_t)(X - 1) * Z);
    dump_dev("fwd_vz", d_vz, (size_t)X * (Z - 1));
    dump_dev("fwd_pl1", d_pl1, npml * Z); dump_dev("fwd_pl2", d_pl2, npml * Z);
    dump_dev("fwd_pr1", d_pr1, npml * Z); dump_dev("fwd_pr2", d_pr2, npml * Z);
    dump_dev("fwd_pt1", d_pt1, npml * nxl); dump_dev("fwd_pt2", d_pt2, npml * nxl);
    dump_dev("fwd_pb1", d_pb1, npml * nxl); dump_dev("fwd_pb2", d_pb2, npml * nxl);
    dump_dev("fwd_gather", d_gather, (size_t)nsteps * nxl);
    dump_dev("strip_vx_last", d_svx + lv * (nsteps - 1), lv);
    dump_dev("strip_vz_last", d_svz + lh * (nsteps - 1), lh);
    dump_dev("strip_plr_last", d_splr + lv * (nsteps - 1), lv);
    dump_dev("strip_ptb_last", d_sptb + lh * (nsteps - 1), lh);

    // reconstruction (rtm_model.cu:367-372, 421-437), nback iterations from it = nsteps-2
    float *d_ps = dalloc<float>((size_t)X * Z), *d_vxs = dalloc<float>((size_t)(X - 1) * Z), *d_vzs = dalloc<float>((size_t)X * (Z - 1));
    cudaMemcpy(d_ps, d_p, sizeof(float) * X * Z, cudaMemcpyDeviceToDevice);
    float *d_bvx = dalloc<float>(lv), *d_bvz = dalloc<float>(lh), *d_bplr = dalloc<float>(lv), *d_bptb = dalloc<float>(lh);
    for (int it = nsteps - 2; it >= nsteps - 1 - nback; it--) {
        cudaMemcpy(d_bvx, d_svx + lv * (it + 1), lv * 4, cudaMemcpyDeviceToDevice);
        cudaMemcpy(d_bvz, d_svz + lh * (it + 1), lh * 4, cudaMemcpyDeviceToDevice);
        read_d_vxpml<<<gpmllr, bpmllr>>>(d_vxs, d_bvx, X, Z, npml);
        read_d_vzpml<<<gpmltb, bpmltb>>>(d_vzs, d_bvz, X, Z, npml);
        cuda_backward_vx<<<gvxb, blk>>>(d_ps, d_vxs, d_rho, d_coef, _dtx, npml, X, Z);
        cuda_backward_vz<<<gvzb, blk>>>(d_ps, d_vzs, d_rho, d_coef, _dtz, npml, X, Z);
        cudaMemcpy(d_bplr, d_splr + lv * it, lv * 4, cudaMemcpyDeviceToDevice);
        cudaMemcpy(d_bptb, d_sptb + lh * it, lh * 4, cudaMemcpyDeviceToDevice);
        read_d_ppmllr<<<gpmllr, bpmllr>>>(d_ps, d_bplr, X, Z, npml);
        read_d_ppmltb<<<gpmltb, bpmltb>>>(d_ps, d_bptb, X, Z, npml);
        cuda_backward_p<<<gp, blk>>>(d_ps, d_vxs, d_vzs, d_rho, d_vp, d_coef, _dtx, _dtz, npml, X, Z);
        cuda_add_source<<<gfull, blk>>>(d_ps, d_src, d_w, dt, 2, X, Z, it);
    }
    ck("backward steps");
    dump_dev("bwd_ps", d_ps, (size_t)X * Z);
    dump_dev("bwd_vxs", d_vxs, (size_t)(X - 1) * Z);
    dump_dev("bwd_vzs", d_vzs, (size_t)X * (Z - 1));
    float meta[12] = {(float)nxl, (float)nzl, (float)npml, dx, dz, dt, fdom, (float)nt,
                      (float)nsx, (float)nsz, amp, alp};
    dump_host("units_meta", meta, 12);
    float meta2[4] = {vpmax, vpmax_prof, (float)nsteps, (float)nback};
    dump_host("units_meta2", meta2, 4);
    std::printf("units done\n");
    return 0;
}

// ---------------------------------------------------------------------------------------
struct RtmCase {
    const char *name;
    int layout, mode, medium_flag, ismth, nshot, nx, nz, nt, npml, smooth_model;
    float dx, dt, fdom, spx0, spz0, dspx, offset, offsetmax, amp, alp, direct, direct0;
    const char *data_from;   // mode 1: directory holding seisReal/ from a mode-0 case
};

static int run_rtm_case(const RtmCase &c)
{
    std::string dir = g_dir + "/" + c.name;
    mkdir_p(dir);
    mkdir_p(dir + "/seisReal");
    mkdir_p(dir + "/output");
    if (c.data_from) {
        for (int s = 1; s <= c.nshot; s++) {
            std::string src = g_dir + "/" + c.data_from + "/seisReal/" + std::to_string(s) + "seisreal.su";
            std::string dst = dir + "/seisReal/" + std::to_string(s) + "seisreal.su";
            FILE *fi = std::fopen(src.c_str(), "rb"), *fo = std::fopen(dst.c_str(), "wb");
            if (!fi || !fo) { std::fprintf(stderr, "copy %s failed\n", src.c_str()); return 4; }
            char buf[65536];
            size_t n;
            while ((n = std::fread(buf, 1, sizeof(buf), fi)) > 0) std::fwrite(buf, 1, n, fo);
            std::fclose(fi); std::fclose(fo);
        }
    }
    const int nx = c.nx, nz = c.nz;
    std::vector<float> vp(nx * nz), rho(nx * nz), diffcoef(100), wavelet(c.nt);
    make_model(nx, nz, c.dx, vp.data(), rho.data(), 0);
    if (c.smooth_model) velsmooth1d(vp.data(), nz, nx, c.smooth_model);   // migration model
    coef_table(diffcoef.data());
    Ricker(wavelet.data(), c.fdom, c.nt, c.dt, 1);
    std::vector<std::vector<float>> img(10, std::vector<float>(nx * nz, 0.0f));
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return 5;
    if (chdir(dir.c_str()) != 0) return 5;
    g_dir = ".";
    dump_host("vp0", vp.data(), vp.size());
    dump_host("rho0", rho.data(), rho.size());
    rtm_model(0, c.nshot, 1, 1, c.mode, c.medium_flag, c.layout, 0, 0, c.ismth, nx, nz, c.nt, c.dx,
              c.dx, c.dt, c.npml, c.direct, c.direct0, 0.25f, c.fdom, c.spx0, c.spz0, c.dspx,
              c.offset, c.offsetmax, c.amp, c.alp, vp.data(), rho.data(), diffcoef.data(),
              wavelet.data(), img[0].data(), img[1].data(), img[2].data(), img[3].data(),
              img[4].data(), img[5].data(), img[6].data(), img[7].data(), img[8].data(),
              img[9].data());
    ck(c.name);
    const char *names[10] = {"image1", "image2s", "image3s", "image4s", "image5s",
                             "image2m", "image3m", "image4m", "image5m", "illum"};
    for (int i = 0; i < 10; i++) dump_host(names[i], img[i].data(), img[i].size());
    if (chdir(cwd) != 0) return 5;
    std::printf("case %s done\n", c.name);
    return 0;
}

static int run_rtm(const std::string root)
{
    //            name      lay mode mf ism nsh  nx  nz   nt npml sm   dx     dt    fdom  spx0   spz0  dspx  off  offmax amp  alp   direct direct0 data_from
    RtmCase B = {"caseB",   2,  0,   0, 0,  2,   96, 64,  600, 32, 0,  10.f, 1e-3f, 25.f, 300.f, 20.f, 360.f, 0.f, 0.f,  1.f, 0.1f, 1.5f, 0.05f, nullptr};
    RtmCase C = {"caseC",   2,  1,   0, 0,  2,   96, 64,  600, 32, 4,  10.f, 1e-3f, 25.f, 300.f, 20.f, 360.f, 0.f, 0.f,  1.f, 0.1f, 1.5f, 0.05f, "caseB"};
    RtmCase D = {"caseD",   1,  0,   1, 2,  2,   96, 64,  500, 32, 0,  10.f, 1e-3f, 25.f, 200.f, 20.f, 550.f, 0.f, 860.f, 1.f, 0.07f, 1.5f, 0.0f, nullptr};
    int rc;
    g_dir = root; if ((rc = run_rtm_case(B))) return rc;
    g_dir = root; if ((rc = run_rtm_case(C))) return rc;
    g_dir = root; if ((rc = run_rtm_case(D))) return rc;
    return 0;
}

// Larger parity-size runs, timed by the reference's own per-shot cudaEvent printout.
static int run_time(const std::string root, const std::string which)
{
    RtmCase T1 = {"time_cfg1", 2, 0, 0, 0, 1, 416, 224, 2000, 32, 0, 10.f, 1e-3f, 20.f, 2000.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.1f, 1.5f, 0.0f, nullptr};
    RtmCase T1b = {"time_cfg1_mig", 2, 1, 0, 0, 1, 416, 224, 2000, 32, 0, 10.f, 1e-3f, 20.f, 2000.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.1f, 1.5f, 0.0f, "time_cfg1"};
    RtmCase T2 = {"time_cfg2", 2, 0, 0, 0, 1, 1696, 352, 4000, 32, 0, 12.5f, 1e-3f, 15.f, 625.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.08f, 1.5f, 0.0f, nullptr};
    RtmCase T2b = {"time_cfg2_mig", 2, 1, 0, 0, 1, 1696, 352, 4000, 32, 0, 12.5f, 1e-3f, 15.f, 625.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.08f, 1.5f, 0.0f, "time_cfg2"};
    int rc;
    if (which == "cfg1" || which == "all") {
        g_dir = root; if ((rc = run_rtm_case(T1))) return rc;
        g_dir = root; if ((rc = run_rtm_case(T1b))) return rc;
    }
    if (which == "cfg2" || which == "all") {
        g_dir = root; if ((rc = run_rtm_case(T2))) return rc;
        g_dir = root; if ((rc = run_rtm_case(T2b))) return rc;
    }
    return 0;
}

// ---------------------------------------------------------------------------------------
// Real-data path.  Model grid dx = 10 m (nx 192, nz 64, nt 600 at 1 ms); data grid dx0 = 20 m,
// nt0 = 300 at 2 ms, so every shot goes through the F-K (x2) and sinc (x2) interpolation.
// Shots at sx = 0, 400, 800 m, 46 receivers from 50 m offset every 20 m: nxlength = 96,
// noffset = 5, 91 migrated traces, 46 data traces; nxlength, nz, nxpad, nzpad are multiples
// of 32.  Data: three hyperbolic 20 Hz Ricker events.
static const int kRealShots = 3, kRealTraces = 46, kRealNt0 = 300;
static const float kRealDx0 = 20.f, kRealDt0 = 2e-3f, kRealOffset = 50.f;

static void put_i32(unsigned char *h, int off, int v) { std::memcpy(h + off, &v, 4); }
static void put_i16(unsigned char *h, int off, short v) { std::memcpy(h + off, &v, 2); }

static int write_real_file(const std::string &path)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return 4;
    std::vector<unsigned char> vol(3600, 0);
    std::fwrite(vol.data(), 1, 3600, f);
    const float t0s[3] = {0.12f, 0.28f, 0.45f}, amps[3] = {1.0f, -0.6f, 0.4f};
    std::vector<float> tr(kRealNt0);
    int itr = 1;
    for (int s = 0; s < kRealShots; s++) {
        const int sx = 400 * s;
        for (int j = 0; j < kRealTraces; j++) {
            const float h = kRealOffset + j * kRealDx0;
            unsigned char hd[240];
            std::memset(hd, 0, sizeof(hd));
            put_i32(hd, 0, itr++);
            put_i32(hd, 12, j + 1);
            put_i32(hd, 36, (int)h);
            put_i32(hd, 72, sx);
            put_i32(hd, 80, sx + (int)h);
            put_i16(hd, 114, (short)kRealNt0);
            put_i16(hd, 116, (short)2000);
            float d2 = kRealDx0;
            std::memcpy(hd + 188, &d2, 4);
            put_i32(hd, 208, kRealTraces);
            std::fwrite(hd, 1, 240, f);
            for (int it = 0; it < kRealNt0; it++) {
                double t = it * (double)kRealDt0, v = 0.0;
                for (int e = 0; e < 3; e++) {
                    double te = std::sqrt((double)t0s[e] * t0s[e] + (h / 2000.0) * (h / 2000.0));
                    double a = M_PI * 20.0 * (t - te);
                    v += amps[e] * (1.0 - 2.0 * a * a) * std::exp(-a * a);
                }
                tr[it] = (float)v;
            }
            std::fwrite(tr.data(), sizeof(float), kRealNt0, f);
        }
    }
    std::fclose(f);
    return 0;
}

static int run_real(const std::string root)
{
    std::string dir = root + "/real";
    mkdir_p(dir);
    mkdir_p(dir + "/seisReal");
    mkdir_p(dir + "/output");
    int rc = write_real_file(dir + "/seisReal/real.sgy");
    if (rc) return rc;
    const int nx = 192, nz = 64, nt = 600, npml = 32;
    const float dx = 10.f, dt = 1e-3f;
    std::vector<float> vp(nx * nz), rho(nx * nz), diffcoef(100), wavelet(nt);
    make_model(nx, nz, dx, vp.data(), rho.data(), 0);
    coef_table(diffcoef.data());
    Ricker(wavelet.data(), 20.f, nt, dt, 1);
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return 5;
    if (chdir(dir.c_str()) != 0) return 5;
    g_dir = ".";
    dump_host("vp0", vp.data(), vp.size());
    dump_host("rho0", rho.data(), rho.size());
    const int nshotall = kRealShots + 2;   // room for a trailing entry
    std::vector<int> prof(4 * nshotall, -7);
    int *rows[4] = {&prof[0], &prof[nshotall], &prof[2 * nshotall], &prof[3 * nshotall]};
    char fname[40] = "real.sgy";
    int endianflag = -1;
    scanshotgather(fname, rows, 1, &endianflag);
    dump_host("profile", prof.data(), prof.size());
    dump_host("endianflag", &endianflag, 1);
    std::vector<std::vector<float>> img(10, std::vector<float>(nx * nz, 0.0f));
    rtm_real(0, kRealShots, 1, 1, /*medium_flag*/ 1, /*flag_layout*/ 3, /*sgyflag*/ 1, endianflag, /*ismth*/ 2,
             nx, nz, nt, dx, dx, dt, nx / 2, nz / 2, kRealNt0, kRealDx0, kRealDx0, kRealDt0, npml, 2, 2,
             /*tsnap*/ 1.0f, /*fdom*/ 20.f, /*spz0*/ 20.f, /*amp*/ 1.f, /*alp*/ 0.1f, /*direct*/ 1.5f,
             /*direct0*/ 0.05f, vp.data(), rho.data(), diffcoef.data(), wavelet.data(), fname, rows,
             img[0].data(), img[1].data(), img[2].data(), img[3].data(), img[4].data(), img[5].data(),
             img[6].data(), img[7].data(), img[8].data(), img[9].data());
    ck("rtm_real");
    const char *names[10] = {"image1", "image2s", "image3s", "image4s", "image5s",
                             "image2m", "image3m", "image4m", "image5m", "illum"};
    for (int i = 0; i < 10; i++) dump_host(names[i], img[i].data(), img[i].size());
    if (chdir(cwd) != 0) return 5;
    std::printf("real done\n");
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s units|rtm|time|real <outdir> [case]\n", argv[0]);
        return 1;
    }
    std::string mode = argv[1];
    g_dir = argv[2];
    mkdir_p(g_dir);
    cudaSetDevice(0);
    if (mode == "units") return run_units();
    if (mode == "rtm") return run_rtm(g_dir);
    if (mode == "time") return run_time(g_dir, argc > 3 ? argv[3] : "cfg1");
    if (mode == "real") return run_real(g_dir);
    return 1;
}
