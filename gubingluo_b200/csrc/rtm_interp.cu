// rtm_interp.cu — resampling of recorded shot gathers onto the modelling grid, on the GPU
// (reference Interpseis2d / GeneralFKinterp / Sincinterp, Interp_function.cpp:10-264, which
// run on the host with FFTW).  Used by the real-data path before the direct-wave mute.
//
//   x: general F-K interpolation by lx = (nx-1)/(nx0-1): cuFFT double-complex transforms
//      (the reference's FFTW plans are double precision) around four kernels;
//   t: 21-tap Kaiser-windowed sinc, one thread per output sample.
//
// Expressions follow the reference's float/double evaluation; products and sums that the
// reference evaluates without fused multiply-add use __fmul_rn/__fadd_rn (float) and
// __dmul_rn/__dadd_rn (double), so only the FFTs themselves round differently.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "rtm_b200.h"
#include "rtm_internal.h"

namespace rtm {

namespace {

constexpr int kTaps = 21;
struct Kaiser21 {
    float w[kTaps];
};

// modZeroBessel / Kaiser (Interp_function.cpp:10-43): 20-term I0 series in double.
double bessel_i0(double x)
{
    double x_2 = x / 2, num = 1, fact = 1, result = 1;
    for (int i = 1; i < 20; i++) {
        num *= x_2 * x_2;
        fact *= i;
        result += num / (fact * fact);
    }
    return result;
}

Kaiser21 kaiser_window()
{
    Kaiser21 k;
    const double m_2 = (double)(kTaps - 1) / 2.0, denom = bessel_i0(2.0);
    for (int n = 0; n < kTaps; n++) {
        double v = (n - m_2) / m_2;
        v = 1 - v * v;
        k.w[n] = (float)(bessel_i0(2.0 * std::sqrt(v)) / denom);
    }
    return k;
}

// Sinc (Interp_function.cpp:44-52): sin(pi x)/(pi x) with the reference's double pi.
__device__ __forceinline__ float sinc_f(float x)
{
    if (x == 0.0f) return 1.0f;
    const double px = 3.1415926535897932 * (double)x;
    return (float)(sin(px) / px);
}

// Sincinterp: out [nt][nx] from in [nt0][ld_in].  Window start it0 - 10 around
// it0 = (int)((it+1)*dt/dt0), sinc centred on it*dt, taps cut at the ends as the reference
// does (at the start the window shifts with the cut, at the end it keeps its first taps).
// The sinc values and window taps depend on the output sample's time only: each block of
// kSincRows rows x 32 traces evaluates them once per row into shared memory (the reference
// evaluates them per trace), then every thread forms (trace * sinc) * window tap by tap.
constexpr int kSincRows = 8;
__global__ void __launch_bounds__(32 * kSincRows) k_sinc(const float *__restrict__ in, int ld_in, float *__restrict__ out,
                                                         int nx, int nt, int nt0, float dt, float dt0, Kaiser21 kw)
{
    __shared__ float s_sinc[kSincRows][kTaps], s_win[kSincRows][kTaps];
    __shared__ int s_start[kSincRows], s_len[kSincRows];
    const int halfnw = 10;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid < kSincRows * kTaps) {
        const int r = tid / kTaps, ik = tid % kTaps;
        const int it = blockIdx.y * kSincRows + r;
        if (it < nt) {
            const int it0 = (int)__fdiv_rn(__fmul_rn((float)(it + 1), dt), dt0);
            const int itstart = max(0, it0 - halfnw), itend = min(nt0 - 1, it0 + halfnw);
            const int lenit = itend - itstart + 1;
            const int inwstart = itstart <= halfnw ? kTaps - lenit : 0;
            if (ik == 0) {
                s_start[r] = itstart;
                s_len[r] = lenit;
            }
            if (ik < lenit) {
                const float t = __fmul_rn((float)it, dt);
                const float tn = __fmul_rn((float)(ik + itstart), dt0);
                s_sinc[r][ik] = sinc_f(__fdiv_rn(__fsub_rn(t, tn), dt0));
                s_win[r][ik] = kw.w[ik + inwstart];
            }
        }
    }
    __syncthreads();
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = threadIdx.y;
    const int it = blockIdx.y * kSincRows + r;
    if (ix >= nx || it >= nt) return;
    const int itstart = s_start[r], lenit = s_len[r];
    float sum = 0.0f;
    for (int ik = 0; ik < lenit; ik++) {
        const float a = in[(size_t)(ik + itstart) * ld_in + ix];
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(a, s_sinc[r][ik]), s_win[r][ik]));
    }
    out[(size_t)it * nx + ix] = sum;
}

// F-K step 1: K [nx0][nt0] and S [Nx][Nt] (zero-padded) from the gather [nt0][nx0].
__global__ void k_fk_load(const float *__restrict__ in, double2 *__restrict__ K, double2 *__restrict__ S, int nx0,
                          int nt0, int Nx, int Nt)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Nx * Nt) return;
    const int ix = (int)(i / Nt), it = (int)(i % Nt);
    double v = 0.0;
    if (ix < nx0 && it < nt0) {
        v = (double)in[(size_t)it * nx0 + ix];
        K[(size_t)ix * nt0 + it] = make_double2(v, 0.0);
    }
    S[i] = make_double2(v, 0.0);
}

// |z| as the reference's fftw_fabs: sqrtf of the float-rounded double re^2 + im^2.
__device__ __forceinline__ float cabs_f(double re, double im)
{
    return sqrtf(__double2float_rn(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im))));
}

// F-K step 2a: Z [nx0][Nt] = (sum of the lx aliased rows of S) / lx, and max |Z| (the lx
// copies of Z that the reference keeps are identical).  Non-negative floats order like
// their bit patterns, so the maximum is an atomicMax on the bits.
__global__ void k_fk_fold(const double2 *__restrict__ S, double2 *__restrict__ Z, unsigned *__restrict__ zmax_bits,
                          int nx0, int Nt, int lx)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float m = 0.0f;
    if (i < (size_t)nx0 * Nt) {
        const int ix = (int)(i / Nt), it = (int)(i % Nt);
        double zr = 0.0, zi = 0.0;
        for (int il = 0; il < lx; il++) {
            const double2 s = S[(size_t)(ix + il * nx0) * Nt + it];
            zr = __dadd_rn(zr, s.x);
            zi = __dadd_rn(zi, s.y);
        }
        zr = __ddiv_rn(zr, (double)lx);
        zi = __ddiv_rn(zi, (double)lx);
        Z[i] = make_double2(zr, zi);
        m = cabs_f(zr, zi);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(zmax_bits, __float_as_uint(m));
}

// F-K step 2b/3a: H = S / (Z + max|Z|*1e-5), |H| > lx^2 -> lx; G1 [nf][Nx] = H * K (K repeated
// lx times along x).
__global__ void k_fk_filter(const double2 *__restrict__ S, const double2 *__restrict__ Z,
                            const double2 *__restrict__ K, const unsigned *__restrict__ zmax_bits,
                            double2 *__restrict__ G1, int nx0, int nt0, int Nx, int Nt, int nf, int lx)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Nx * nf) return;
    const int it = (int)(i / Nx), ix = (int)(i % Nx);
    const int ib = ix % nx0;
    const double eps = __dmul_rn((double)__uint_as_float(*zmax_bits), 0.00001);
    const double2 s = S[(size_t)ix * Nt + it];
    double2 z = Z[(size_t)ib * Nt + it];
    z.x = __dadd_rn(z.x, eps);
    const double den = __dadd_rn(__dmul_rn(z.x, z.x), __dmul_rn(z.y, z.y));
    double h0 = __ddiv_rn(__dadd_rn(__dmul_rn(s.x, z.x), __dmul_rn(s.y, z.y)), den);
    double h1 = __ddiv_rn(__dsub_rn(__dmul_rn(s.y, z.x), __dmul_rn(s.x, z.y)), den);
    if (cabs_f(h0, h1) > (float)(lx * lx)) {
        h0 = (double)(float)lx;
        h1 = 0.0;
    }
    const double2 c = K[(size_t)ib * nt0 + it];
    G1[i] = make_double2(__dsub_rn(__dmul_rn(h0, c.x), __dmul_rn(h1, c.y)),
                         __dadd_rn(__dmul_rn(h0, c.y), __dmul_rn(h1, c.x)));
}

// F-K step 3b: G [nx][nt0] from G1 [nf][Nx] (after the inverse transform along x): the
// first nf frequencies as they are, the rest the conjugate of G1 at it1 = (nt0+1)/2 - (it-nf)
// (mirror 0, the reference's indexing) or at nt0 - it (mirror 1, the Hermitian partner).
// For odd nt0 under mirror 0 the first it1 is nf, one row past G1; it reads as zero.
__global__ void k_fk_mirror(const double2 *__restrict__ G1, double2 *__restrict__ G, int nx, int nt0, int Nx, int nf,
                            int mirror)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nx * nt0) return;
    const int ix = (int)(i / nt0), it = (int)(i % nt0);
    double2 g = make_double2(0.0, 0.0);
    if (it < nf) {
        g = G1[(size_t)it * Nx + ix];
    } else {
        const int src = mirror ? nt0 - it : (nt0 + 1) / 2 - (it - nf);
        if (src < nf) {
            g = G1[(size_t)src * Nx + ix];
            g.y = -g.y;
        }
    }
    G[i] = g;
}

// F-K step 3c: out [rows][nx] = real part of G [nx][nt0] (after the inverse transform along t).
__global__ void k_fk_store(const double2 *__restrict__ G, float *__restrict__ out, int nx, int nt0, int rows)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)rows * nx) return;
    const int it = (int)(i / nx), ix = (int)(i % nx);
    out[i] = __double2float_rn(G[(size_t)ix * nt0 + it].x);
}

unsigned blocks_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

#define CKI(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(RTM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)
#define CKF(call)                                                                                   \
    do {                                                                                            \
        cufftResult r_ = (call);                                                                    \
        if (r_ != CUFFT_SUCCESS) return fail(RTM_ERR_CUDA, std::string(#call) + " failed, cufft " + std::to_string((int)r_)); \
    } while (0)

void InterpPlan::release()
{
    if (plans) {
        cufftDestroy((cufftHandle)p_k);
        cufftDestroy((cufftHandle)p_s);
        cufftDestroy((cufftHandle)p_x);
        cufftDestroy((cufftHandle)p_t);
    }
    if (work) cudaFree(work);
    *this = InterpPlan();
}

int interp_check_guards(const InterpPlan &p)
{
    std::vector<unsigned char> h;
    for (const auto &g : p.guards) {
        h.resize(g.second);
        CKI(cudaMemcpy(h.data(), (char *)p.work + g.first, g.second, cudaMemcpyDeviceToHost));
        for (unsigned char c : h)
            if (c != 0xA5) return fail(RTM_ERR_CUDA, "device write past the end of a resampling buffer");
    }
    return RTM_OK;
}

int interp_shape(int nx0, int nt0, int nx, int nt, InterpShape &sh)
{
    std::memset(&sh, 0, sizeof(sh));
    if (nx0 < 1 || nt0 < 1 || nx < 1 || nt < 1) return fail(RTM_ERR_ARG, "interpolation sizes must be positive");
    sh.nx0 = nx0; sh.nt0 = nt0; sh.nx = nx; sh.nt = nt;
    sh.fk = nx > nx0;
    sh.sinc = nt > nt0;
    if (sh.fk) {
        if (nx0 < 2) return fail(RTM_ERR_ARG, "F-K interpolation needs at least two recorded traces");
        sh.lx = (nx - 1) / (nx0 - 1);
        sh.Nx = sh.lx * nx0;
        sh.Nt = sh.lx * nt0;
        sh.nf = 1 + nt0 / 2;
        if (nx > sh.Nx)
            return fail(RTM_ERR_ARG, "F-K interpolation: " + std::to_string(nx) + " output traces exceed lx*nx0 = " +
                                         std::to_string(sh.Nx));
    }
    return RTM_OK;
}

// Device workspace and cuFFT plans for one interpolation shape (kept while the shape repeats).
static int plan_for(InterpPlan &p, const InterpShape &sh, cudaStream_t st)
{
    if (p.work && std::memcmp(&p.shape, &sh, sizeof(sh)) == 0 && (!sh.fk || p.plans)) {
        if (p.plans) {
            CKF(cufftSetStream((cufftHandle)p.p_k, st));
            CKF(cufftSetStream((cufftHandle)p.p_s, st));
            CKF(cufftSetStream((cufftHandle)p.p_x, st));
            CKF(cufftSetStream((cufftHandle)p.p_t, st));
        }
        return RTM_OK;
    }
    p.release();
    p.shape = sh;
    size_t off = 0;
    const char *gv = std::getenv("RTM_B200_GUARDS");
    const bool guard = gv && std::atoi(gv) != 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        if (guard) {
            p.guards.push_back({o + bytes, off + 256 - (o + bytes)});
            off += 256;
        }
        return o;
    };
    const size_t o_in = take(sizeof(float) * (size_t)sh.nt0 * sh.nx0);
    size_t o_tmp = 0, o_K = 0, o_S = 0, o_Z = 0, o_G1 = 0, o_G = 0, o_zm = 0;
    if (sh.fk) {
        o_tmp = take(sizeof(float) * (size_t)sh.nt0 * sh.nx);
        o_K = take(sizeof(double2) * (size_t)sh.nx0 * sh.nt0);
        o_S = take(sizeof(double2) * (size_t)sh.Nx * sh.Nt);
        o_Z = take(sizeof(double2) * (size_t)sh.nx0 * sh.Nt);
        o_G1 = take(sizeof(double2) * (size_t)sh.nf * sh.Nx);
        o_G = take(sizeof(double2) * (size_t)sh.nx * sh.nt0);
        o_zm = take(sizeof(unsigned));
    }
    CKI(cudaMalloc(&p.work, off));
    char *b = (char *)p.work;
    for (const auto &g : p.guards) CKI(cudaMemsetAsync(b + g.first, 0xA5, g.second, st));
    p.d_in = (float *)(b + o_in);
    if (sh.fk) {
        p.d_tmp = (float *)(b + o_tmp);
        p.K = b + o_K;
        p.S = b + o_S;
        p.Z = b + o_Z;
        p.G1 = b + o_G1;
        p.G = b + o_G;
        p.zmax = (unsigned *)(b + o_zm);
        cufftHandle h[4];
        int made = 0;
        int n_x[1] = {sh.Nx}, n_t[1] = {sh.nt0};
        cufftResult r = cufftPlan2d(&h[0], sh.nx0, sh.nt0, CUFFT_Z2Z);
        if (r == CUFFT_SUCCESS && ++made) r = cufftPlan2d(&h[1], sh.Nx, sh.Nt, CUFFT_Z2Z);
        if (r == CUFFT_SUCCESS && ++made)
            r = cufftPlanMany(&h[2], 1, n_x, nullptr, 1, sh.Nx, nullptr, 1, sh.Nx, CUFFT_Z2Z, sh.nf);
        if (r == CUFFT_SUCCESS && ++made)
            r = cufftPlanMany(&h[3], 1, n_t, nullptr, 1, sh.nt0, nullptr, 1, sh.nt0, CUFFT_Z2Z, sh.nx);
        if (r == CUFFT_SUCCESS) made++;
        if (made < 4) {
            for (int i = 0; i < made; i++) cufftDestroy(h[i]);
            return fail(RTM_ERR_CUDA, "cuFFT plan creation failed, cufft " + std::to_string((int)r));
        }
        p.p_k = h[0];
        p.p_s = h[1];
        p.p_x = h[2];
        p.p_t = h[3];
        p.plans = true;
        CKF(cufftSetStream((cufftHandle)p.p_k, st));
        CKF(cufftSetStream((cufftHandle)p.p_s, st));
        CKF(cufftSetStream((cufftHandle)p.p_x, st));
        CKF(cufftSetStream((cufftHandle)p.p_t, st));
    }
    return RTM_OK;
}

// Interpseis2d on the device: p.d_in [nt0][nx0] (already uploaded) -> out [nt][nx].  The
// branches where the reference's result is undefined are defined as in the restatement
// the tests check against: with neither x nor t interpolation the first nt samples of the
// first nx traces are copied, and the x-only branch keeps the first nt of its nt0 rows.
static int interp_run(InterpPlan &p, float *out, float dt, float dt0, int mirror, cudaStream_t st, int *launches)
{
    const InterpShape &sh = p.shape;
    const int T = 256;
    const float *src = p.d_in;
    int ld = sh.nx0;
    if (sh.fk) {
        double2 *K = (double2 *)p.K, *S = (double2 *)p.S, *Z = (double2 *)p.Z, *G1 = (double2 *)p.G1,
                *G = (double2 *)p.G;
        CKI(cudaMemsetAsync(p.zmax, 0, sizeof(unsigned), st));
        k_fk_load<<<blocks_for((size_t)sh.Nx * sh.Nt, T), T, 0, st>>>(p.d_in, K, S, sh.nx0, sh.nt0, sh.Nx, sh.Nt);
        CKF(cufftExecZ2Z((cufftHandle)p.p_k, (cufftDoubleComplex *)K, (cufftDoubleComplex *)K, CUFFT_FORWARD));
        CKF(cufftExecZ2Z((cufftHandle)p.p_s, (cufftDoubleComplex *)S, (cufftDoubleComplex *)S, CUFFT_FORWARD));
        k_fk_fold<<<blocks_for((size_t)sh.nx0 * sh.Nt, T), T, 0, st>>>(S, Z, p.zmax, sh.nx0, sh.Nt, sh.lx);
        k_fk_filter<<<blocks_for((size_t)sh.Nx * sh.nf, T), T, 0, st>>>(S, Z, K, p.zmax, G1, sh.nx0, sh.nt0, sh.Nx,
                                                                            sh.Nt, sh.nf, sh.lx);
        CKF(cufftExecZ2Z((cufftHandle)p.p_x, (cufftDoubleComplex *)G1, (cufftDoubleComplex *)G1, CUFFT_INVERSE));
        k_fk_mirror<<<blocks_for((size_t)sh.nx * sh.nt0, T), T, 0, st>>>(G1, G, sh.nx, sh.nt0, sh.Nx, sh.nf, mirror);
        CKF(cufftExecZ2Z((cufftHandle)p.p_t, (cufftDoubleComplex *)G, (cufftDoubleComplex *)G, CUFFT_INVERSE));
        const int rows = sh.sinc ? sh.nt0 : std::min(sh.nt, sh.nt0);
        float *dst = sh.sinc ? p.d_tmp : out;
        k_fk_store<<<blocks_for((size_t)rows * sh.nx, T), T, 0, st>>>(G, dst, sh.nx, sh.nt0, rows);
        if (launches) *launches += 5;
        src = p.d_tmp;
        ld = sh.nx;
    }
    if (sh.sinc) {
        dim3 blk(32, kSincRows), grd((sh.nx + 31) / 32, (sh.nt + kSincRows - 1) / kSincRows);
        k_sinc<<<grd, blk, 0, st>>>(src, ld, out, sh.nx, sh.nt, sh.nt0, dt, dt0, kaiser_window());
        if (launches) *launches += 1;
    } else if (!sh.fk) {
        CKI(cudaMemcpy2DAsync(out, sizeof(float) * sh.nx, src, sizeof(float) * ld, sizeof(float) * sh.nx, sh.nt,
                              cudaMemcpyDeviceToDevice, st));
    }
    CKI(cudaGetLastError());
    return RTM_OK;
}

int interp_gather_device(InterpPlan &p, const float *host_in, int nx0, int nt0, float *d_out, int nx, int nt, float dt,
                         float dt0, int mirror, cudaStream_t_fwd st, int *launches)
{
    InterpShape sh;
    int rc = interp_shape(nx0, nt0, nx, nt, sh);
    if (rc) return rc;
    rc = plan_for(p, sh, st);
    if (rc) return rc;
    CKI(cudaMemcpyAsync(p.d_in, host_in, sizeof(float) * (size_t)nt0 * nx0, cudaMemcpyHostToDevice, st));
    return interp_run(p, d_out, dt, dt0, mirror, st, launches);
}

}  // namespace rtm

using namespace rtm;

extern "C" int rtm_interp_gather(const float *seisobs, int nx0, int nt0, float *seiscal, int nx, int nt, float dt,
                                 float dt0, int mirror, int device)
{
    clear_error();
    if (!seisobs || !seiscal) return fail(RTM_ERR_ARG, "rtm_interp_gather: null buffer");
    if (mirror != 0 && mirror != 1) return fail(RTM_ERR_ARG, "rtm_interp_gather: mirror must be 0 or 1");
    InterpShape sh0;
    if (int rc0 = interp_shape(nx0, nt0, nx, nt, sh0)) return rc0;
    CKI(cudaSetDevice(device));
    cudaStream_t st;
    CKI(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    InterpPlan p;
    float *d_out = nullptr;
    int rc = RTM_OK;
    if (cudaMalloc(&d_out, sizeof(float) * (size_t)nt * nx) != cudaSuccess)
        rc = fail(RTM_ERR_NOMEM, "rtm_interp_gather: device allocation failed");
    if (!rc) rc = interp_gather_device(p, seisobs, nx0, nt0, d_out, nx, nt, dt, dt0, mirror, st, nullptr);
    if (!rc && cudaStreamSynchronize(st) == cudaSuccess) rc = interp_check_guards(p);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(seiscal, d_out, sizeof(float) * (size_t)nt * nx, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(RTM_ERR_CUDA, std::string("rtm_interp_gather: ") + cudaGetErrorString(e));
    }
    p.release();
    if (d_out) cudaFree(d_out);
    cudaStreamDestroy(st);
    return rc;
}
