// rtm_gpu_main.cpp — drop-in replacement of the reference's rtm_gpu program
// (gubingluo RTM_GPU_velstr.cpp:37-317): reads ./input/cmd.in and the parameter file it
// names, reads and regrids the velocity (and density) model, prints the same parameter
// banner, migrates through rtm_model() (modelled data) or rtm_real() (a recorded multi-shot
// file, dataflag 1) and writes ./output/{idevice}*.su.
// Run with "--help" for the parameter-file layout (the reference's README promises a
// selfdoc that its program does not print).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rtm_b200.h"

static void selfdoc()
{
    std::printf(
        "rtm_gpu: 2D acoustic prestack reverse-time migration on one B200 GPU.\n"
        "Reads ./input/cmd.in; its second line names the parameter file in ./input/.\n"
        "The parameter file alternates one comment line and one value line:\n"
        "  dt0 nt0 tsnap | xmax zmax dx0 dz0 | fdom Amp alp | spx0 spz0 dspx |\n"
        "  offset offsetmax | startshot nshot dshot nshotall | npml |\n"
        "  medium_flag ismth | direct direct0 | idevice | flag_layout (1 bilateral,\n"
        "  2 full array, 3 unilateral right, 4 unilateral left) | mode (0 model the data,\n"
        "  1 data in ./seisReal/) | dataflag | sgyflag | endianflag | rhoflag | vp_file |\n"
        "  [shotgather_file if dataflag] | [rho_file if rhoflag]\n"
        "dataflag 1 migrates the multi-shot SU/SEG-Y file ./seisReal/<shotgather_file>: its shot\n"
        "  table is scanned once into ./shotprofileId.dat (reused when present).\n"
        "Writes ./output/{idevice}{Illum,Image1,Image2s,...,Image5m}.su.\n"
        "Environment: RTM_B200_STRIPS / RTM_B200_GATHERS = fp32|fp16|bf16,\n"
        "  RTM_B200_ACCUM_FP64=1|2|3 (fp64 / compensated fp32 / fp64 totals of 32-step fp32 sums),\n"
        "  RTM_B200_BATCH=<shots per launch>, RTM_B200_RECEIVER_DEPTH=<cells>,\n"
        "  RTM_B200_EXTRA_IMAGES=0|1|2, RTM_B200_FK_MIRROR=0|1, RTM_B200_LOG=<JSON-lines file>.\n"
        "Options: --checkpoint <file> saves the stacked images after every batch;\n"
        "  --resume continues from that file when it matches the run (same parameters and models).\n");
}

int main(int argc, char **argv)
{
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "--help") || !std::strcmp(argv[i], "-h")) {
            selfdoc();
            return 0;
        } else if (!std::strcmp(argv[i], "--checkpoint") && i + 1 < argc) {
            setenv("RTM_B200_CHECKPOINT", argv[++i], 1);
        } else if (!std::strcmp(argv[i], "--resume")) {
            setenv("RTM_B200_RESUME", "1", 1);
        } else {
            std::printf("unknown argument %s\n", argv[i]);
            selfdoc();
            return 1;
        }
    }
    rtm_params P;
    if (rtm_read_params("./input", &P) != RTM_OK) {
        std::printf("%s\n", rtm_last_error());
        selfdoc();
        return 1;
    }
    const int nx0 = (int)(P.xmax / P.dx0) + 1, nz0 = (int)(P.zmax / P.dz0) + 1;   // :121-122
    if (P.spx0 < 0 || P.spz0 < 0 || P.spx0 + (P.nshot - 1) * P.dspx > (nx0 - 1) * P.dx0 ||
        P.spx0 + (P.nshot - 1) * P.dspx < 0) {
        std::printf("the shot position out of the model !\nplease check the parameter !\n");
        return 1;
    }
    std::vector<float> vp0((size_t)nx0 * nz0);
    char path[600];
    std::snprintf(path, sizeof(path), "./input/%s", P.vp_file);
    if (rtm_read_velocity(path, nx0, nz0, vp0.data()) != RTM_OK) {
        std::printf("The file %s open failed !\n", P.vp_file);
        return 1;
    }
    float dx, dz, dt, vpmin, vpmax;
    int nx, nz, nt, lx, lz;
    rtm_get_constant(vp0.data(), P.fdom, P.dx0, P.dz0, nx0, nz0, P.nt0, P.dt0, &dx, &dz, &nx, &nz, &nt, &dt, &lx,
                     &lz, &vpmin, &vpmax);
    std::vector<float> vp((size_t)nx * nz), rho((size_t)nx * nz);
    rtm_interp_model(vp0.data(), vp.data(), nx0, nz0, nx, nz, lx, lz);
    if (P.rhoflag) {   // :140-148 (densities given in g/cc are scaled to kg/m^3)
        std::snprintf(path, sizeof(path), "./input/%s", P.rho_file);
        if (rtm_read_velocity(path, nx0, nz0, vp0.data()) != RTM_OK) {
            std::printf("The file %s open failed !\n", P.rho_file);
            return 1;
        }
        float m = vp0[0];
        for (float v : vp0) m = v > m ? v : m;
        int rhomax = (int)m;
        if (rhomax < 10.0)
            for (float &v : vp0) v *= 1000.0;
        rtm_interp_model(vp0.data(), rho.data(), nx0, nz0, nx, nz, lx, lz);
    } else {
        for (float &v : rho) v = 2000.0f;
    }
    std::printf("=====================================================\n");
    std::printf("=====================================================\n");
    std::printf("Prestack Reverse Time Migration by Bingluo Gu from UPC.\n");
    std::printf("            version 4.0  date 2015.11.25               \n");
    std::printf("        (B200 sm_100a implementation: %s)\n", rtm_version());
    std::printf("=====================================================\n");
    std::printf("=====================================================\n");
    std::printf("================Required parameters:=================\n");
    std::printf(" velfile=   %s\n", P.vp_file);
    std::printf(" nshot  =   %d\t fshot  =   %d\t dshot  =   %d\n", P.nshot, P.startshot, P.dshot);
    std::printf(" nz     =   %d\t nx     =   %d\t nt     =   %d\n", nz0, nx0, P.nt0);
    std::printf(" dz     =   %.1f\t dx     =   %.1f\t dt     =   %.4f\n", P.dz0, P.dx0, P.dt0);
    std::printf(" t      =   %f\n", P.nt0 * P.dt0);
    std::printf(" vmin   =   %.2f\n vmax   =   %.2f\n", vpmin, vpmax);
    std::printf(" fdom      =  %f  dominant frequency\n", P.fdom);
    std::printf(" npml      =  %2d  pml absorb layers number\n", P.npml);
    std::printf(" Norder    =  %2d  order of finite difference\n", 20);
    std::printf(" dataflag  =  %2d  0: model data:                 1: real data\n", P.dataflag);
    std::printf(" mode      =  %2d  0: generate seismic profile;   1: seismic profile exist\n", P.mode);
    std::printf(" format:      %2d  0: su;                         1: sgy\n", P.sgyflag);
    std::printf(" Endian:      %2d  0: little edition;             1: big edition\n", P.endianflag);
    std::printf(" layout:      %2d  1: Bilateral;  2: full array;  3: Unilateral(r);  4: Unilateral(l)\n",
                P.flag_layout);
    std::printf("=================Optional parameters:================\n");
    std::printf(" nz     =   %d\t nx   =   %d\t nt   =   %d\n", nz, nx, nt);
    std::printf(" dz     =   %.1f\t dx   =   %.1f\t dt   =   %.4f\n", dz, dx, dt);
    std::printf(" lz     =   %d\t lx   =   %d\n", lz, lx);
    std::printf(" t      =   %f\n", nt * dt);
    std::printf("=======================================================\n");
    float coef[100];
    rtm_coef_table(coef);
    std::vector<float> wavelet(nt, 0.0f);
    const size_t n = (size_t)nx * nz;
    std::vector<std::vector<float>> img(10, std::vector<float>(n, 0.0f));
    if (!P.dataflag) {
        rtm_model(P.idevice, P.nshot, P.startshot, P.dshot, P.mode, P.medium_flag, P.flag_layout, P.sgyflag,
                  P.endianflag, P.ismth, nx, nz, nt, dx, dz, dt, P.npml, P.direct, P.direct0, P.tsnap, P.fdom,
                  P.spx0, P.spz0, P.dspx, P.offset, P.offsetmax, P.amp, P.alp, vp.data(), rho.data(), coef,
                  wavelet.data(), img[0].data(), img[1].data(), img[2].data(), img[3].data(), img[4].data(),
                  img[5].data(), img[6].data(), img[7].data(), img[8].data(), img[9].data());
    } else {
        // :226-252: the shot table of the recorded file, cached in ./shotprofileId.dat (one
        // "sx ntrace first-trace offset" line per shot); a fresh scan also sets the byte order
        if (P.nshotall < 1) {
            std::printf("nshotall must be >= 1 for real data\n");
            return 1;
        }
        std::vector<int> prof((size_t)4 * P.nshotall, 0);
        int *rows[4] = {&prof[0], &prof[P.nshotall], &prof[2 * (size_t)P.nshotall], &prof[3 * (size_t)P.nshotall]};
        FILE *cache = std::fopen("shotprofileId.dat", "r");
        if (!cache) {
            std::snprintf(path, sizeof(path), "./seisReal/%s", P.shotgather_file);
            int found = rtm_scan_shotgather(path, P.sgyflag, &P.endianflag, prof.data(), P.nshotall);
            if (found < 0) {
                std::printf("rtm_gpu: %s\n", rtm_last_error());
                return 1;
            }
            std::printf("nt %d\n", P.nt0);
            std::printf("shots found: %d\n", found);
            cache = std::fopen("shotprofileId.dat", "w");
            if (cache) {
                for (int i = 0; i < P.nshotall; i++)
                    std::fprintf(cache, "%d %d %d %d\n", rows[0][i], rows[1][i], rows[2][i], rows[3][i]);
                std::fclose(cache);
            }
        } else {
            for (int i = 0; i < P.nshotall; i++)
                if (std::fscanf(cache, "%d %d %d %d", &rows[0][i], &rows[1][i], &rows[2][i], &rows[3][i]) != 4) {
                    std::printf("shotprofileId.dat holds fewer than %d shots\n", P.nshotall);
                    std::fclose(cache);
                    return 1;
                }
            std::fclose(cache);
        }
        char fname[256];
        std::snprintf(fname, sizeof(fname), "%s", P.shotgather_file);
        rtm_real(P.idevice, P.nshot, P.startshot, P.dshot, P.medium_flag, P.flag_layout, P.sgyflag, P.endianflag,
                 P.ismth, nx, nz, nt, dx, dz, dt, nx0, nz0, P.nt0, P.dx0, P.dz0, P.dt0, P.npml, lx, lz, P.tsnap,
                 P.fdom, P.spz0, P.amp, P.alp, P.direct, P.direct0, vp.data(), rho.data(), coef, wavelet.data(),
                 fname, rows, img[0].data(), img[1].data(), img[2].data(), img[3].data(), img[4].data(),
                 img[5].data(), img[6].data(), img[7].data(), img[8].data(), img[9].data());
    }
    if (rtm_last_error()[0]) {
        std::printf("rtm_gpu: %s\n", rtm_last_error());
        return 1;
    }
    // :260-297 (image1, image2s..5s at [0..4], image2m..5m at [5..8], Illum at [9])
    const char *names[10] = {"Image1", "Image2s", "Image3s", "Image4s", "Image5s",
                             "Image2m", "Image3m", "Image4m", "Image5m", "Illum"};
    for (int i = 0; i < 10; i++) {
        std::snprintf(path, sizeof(path), "./output/%d%s.su", P.idevice, names[i]);
        rtm_write_image_su(path, img[i].data(), nz, nx, dz);
    }
    std::printf("The program calculate over !\n");
    return 0;
}
