// kf_noalloc.cu -- the 3-D real-to-complex transform without any device allocation.
//
// kf_fft_r2c runs inside a context whose creation allocates device memory for
// its work buffers.  Some host programs cannot let a library allocate: a host
// that owns a fixed device-memory pool and hands plugins only the buffers it
// has budgeted, or a time-critical loop that must not pay for cudaMalloc's
// latency and implicit device-wide synchronisation.  kf_fft_r2c_noalloc
// serves them: the caller passes the input and output buffers, and the one
// intermediate array of the three-pass transform lives in a file-scope
// static device array (kf_noalloc_scratch below) that the CUDA runtime places
// on every GPU that loads this library and keeps until the process exits.
//
// Limits and sharing: grids of n = 16, 32 or 64 (the scratch holds one
// 64 x 64 x 33 complex-double array plus the twiddle table and the job
// descriptors, 2,166,784 bytes); every call on a device reuses the same array,
// so calls that overlap on that GPU (other streams, other host threads) race
// and must be serialised by the caller.  Each call writes every scratch entry
// it reads before reading it, so nothing has to start at zero.
//
// Set-up: each call outside a stream capture looks up the array's device
// address with cudaGetSymbolAddress (the array's name is only a host-side
// stand-in; handing it to a kernel would fault or silently use the wrong
// memory) and remembers it per device; a call made while its stream is being
// captured uses the remembered address.  Looking it up again on every
// uncaptured call keeps the address right after a cudaDeviceReset, which
// reloads the module (possibly elsewhere).  With lazy module loading (the CUDA
// default since 12.2) the first call on a device also loads this module,
// which places the static array in device memory and synchronises: that first
// call is a warm-up, to be made before the allocation-free part of the
// program and before any stream capture.
//
// An asynchronous error that is already pending when a call starts (from
// earlier, unrelated work) is reported as such and left pending; the call's
// own launch errors are reported as its own.
#include <cmath>
#include <mutex>
#include <string>

#include "../../include/kielflow_b200.h"
#include "kf_passes.cuh"

using namespace kf;

std::string &kf_global_error();  // kf_capi.cu: message for kf_last_error(NULL)

namespace {

constexpr int KF_NOALLOC_MAX_N = 64;
constexpr size_t KF_NOALLOC_GRID_BYTES =
    sizeof(double2) * (size_t)KF_NOALLOC_MAX_N * KF_NOALLOC_MAX_N * (KF_NOALLOC_MAX_N / 2 + 1);
constexpr size_t KF_NOALLOC_TW_OFF = KF_NOALLOC_GRID_BYTES;                     // 64 twiddles
constexpr size_t KF_NOALLOC_JOB_OFF = KF_NOALLOC_TW_OFF + 64 * sizeof(double2);  // job descriptors
constexpr size_t KF_NOALLOC_BYTES = KF_NOALLOC_JOB_OFF + 3072;

}  // namespace

static __device__ __align__(256) unsigned char kf_noalloc_scratch[KF_NOALLOC_BYTES];

namespace {

struct NoallocParams {
    double2 tw[KF_NOALLOC_MAX_N];
    AxisJob ay, ax;
    ZJob z;
};

// Copies the twiddles and job descriptors (kernel parameters) into the
// scratch, so that no host-to-device copy is needed.
__global__ void k_noalloc_setup(NoallocParams p, unsigned char *scratch, int n) {
    double2 *tw = reinterpret_cast<double2 *>(scratch + KF_NOALLOC_TW_OFF);
    for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = p.tw[i];
    if (threadIdx.x == 0) {
        AxisJob *aj = reinterpret_cast<AxisJob *>(scratch + KF_NOALLOC_JOB_OFF);
        aj[0] = p.ay;
        aj[1] = p.ax;
        ZJob *zj = reinterpret_cast<ZJob *>(scratch + KF_NOALLOC_JOB_OFF + 2 * sizeof(AxisJob));
        zj[0] = p.z;
    }
}

std::mutex g_mu;
unsigned char *g_scratch[64] = {};  // per-device address of kf_noalloc_scratch

int fail(int code, const std::string &msg) {
    kf_global_error() = msg;
    return code;
}

template <int N>
cudaError_t run(const double *in, double *out, unsigned char *scratch, cudaStream_t st) {
    NoallocParams p;
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < N; ++m) {  // the table of build_tables in kf_capi.cu, bit for bit
        long double a = twopi * (long double)m / (long double)N;
        p.tw[m] = make_double2((double)cosl(a), (double)(-sinl(a)));
    }
    double2 *mid = reinterpret_cast<double2 *>(scratch);
    p.z = ZJob{in, nullptr, out, nullptr, MUL_NONE, MUL_NONE};      // z: real rows -> half spectra (out)
    p.ay = AxisJob{out, mid, MUL_NONE, 0};                           // y: out -> scratch
    p.ax = AxisJob{mid, out, MUL_NONE, 0};                           // x: scratch -> out
    k_noalloc_setup<<<1, 64, 0, st>>>(p, scratch, N);
    const double2 *tw = reinterpret_cast<const double2 *>(scratch + KF_NOALLOC_TW_OFF);
    const AxisJob *aj = reinterpret_cast<const AxisJob *>(scratch + KF_NOALLOC_JOB_OFF);
    const ZJob *zj = reinterpret_cast<const ZJob *>(scratch + KF_NOALLOC_JOB_OFF + 2 * sizeof(AxisJob));
    constexpr int NZC = N / 2 + 1, LZ = ZTile<double>::LZ, P = Plan<N>::P, TC = Tile<double>::TC;
    const Geo<double> g{N, NZC, nullptr, nullptr, 0.};  // no multipliers: the axis tables are not read
    const int nrows = N * N;
    k_z_r2c<double, N><<<(nrows + LZ - 1) / LZ, LZ * P, ZSmem<double, N, false>::bytes, st>>>(
        zj, 1, nrows, tw);
    const size_t smem = (size_t)N * TC * sizeof(double2);
    k_axis_pass<double, N, -1><<<N * ((NZC + TC - 1) / TC), TC * P, smem, st>>>(aj, 1, 1, g, tw);
    k_axis_pass<double, N, -1><<<(N * NZC + TC - 1) / TC, TC * P, smem, st>>>(aj + 1, 1, 0, g, tw);
    return cudaGetLastError();
}

}  // namespace

extern "C" int kf_fft_r2c_noalloc(int n, const double *in_real, double *out_complex, void *cuda_stream) {
    if (!in_real || !out_complex) return fail(KF_ERR_ARG, "kf_fft_r2c_noalloc: null buffer");
    if (n != 16 && n != 32 && n != 64)
        return fail(KF_ERR_ARG, "kf_fft_r2c_noalloc: n must be 16, 32 or 64 (static scratch holds at most "
                                "64^3; use kf_fft_r2c for larger grids)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(KF_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(KF_ERR_ARG, "kf_fft_r2c_noalloc: device ordinal above 63");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return fail(KF_ERR_CUDA, std::string("kf_fft_r2c_noalloc: an earlier CUDA error is pending (not cleared): ") +
                                     cudaGetErrorString(e));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return fail(KF_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    unsigned char *scratch;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (cap == cudaStreamCaptureStatusNone || !g_scratch[dev]) {
            if (cap != cudaStreamCaptureStatusNone)
                return fail(KF_ERR_ARG, "kf_fft_r2c_noalloc: the first call on a device must not be captured "
                                        "(it looks up the static array's address)");
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, kf_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(KF_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch[dev] = static_cast<unsigned char *>(ptr);
        }
        scratch = g_scratch[dev];
    }
    e = n == 16 ? run<16>(in_real, out_complex, scratch, st)
      : n == 32 ? run<32>(in_real, out_complex, scratch, st)
                : run<64>(in_real, out_complex, scratch, st);
    if (e != cudaSuccess) return fail(KF_ERR_CUDA, std::string("kf_fft_r2c_noalloc: ") + cudaGetErrorString(e));
    return KF_OK;
}
