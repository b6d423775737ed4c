// sg_noalloc.cu -- direct-summation FP64 forces for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured, hosts that hand the GPU's memory to their own pool and
// forbid other allocations, or codes that must not add device allocations
// after start-up.  sphgrav_forces_fp64_noalloc serves them: the caller
// passes device inputs and outputs, and the only other memory the kernels
// use is the file-scope array below, which the CUDA runtime places in every
// GPU that loads this library and keeps there until the process exits.
//
// The kernel is the FP64 direct sum (same pair formulas and branch rule as
// the reference's CPU path, parallel_bleeding_edge/src/cpu_grav.f:46-157)
// on the caller's particle order, without the sorted layout the context API
// builds.  The j-range is split into chunks whose FP64 partial sums go to the
// static scratch; a second kernel adds them in chunk order, so the result is
// deterministic.
#include <algorithm>
#include "sg_launch.h"
#include "../../include/sphgrav_b200.h"

namespace sg {

constexpr int NA_NT = 128;   // rows per block
constexpr int NA_TJ = 128;   // sources staged per shared-memory tile
constexpr size_t NA_SCRATCH_DOUBLES = SPHGRAV_NOALLOC_SCRATCH_BYTES / sizeof(double);

// Partial sums [chunk][4][n].  Every element a call reads was written earlier
// in the same call, so nothing needs clearing between calls.
static __device__ __align__(256) double g_noalloc_scratch[NA_SCRATCH_DOUBLES];

// FP64 pair of rows i and sources j in the caller's order (no sorting):
// H^2 = |range2|, self-potential flag range2 > 0, lower index = min(i, j).
static __device__ __noinline__ PairOut pair_f64_raw(const double *x, const double *y,
                                                    const double *z, const double *m,
                                                    const double *r2in, int nkernel, int i, int j)
{
    const double dr1 = x[j] - x[i], dr2 = y[j] - y[i], dr3 = z[j] - z[i];
    const double r2 = SG_A(SG_A(SG_M(dr1, dr1), SG_M(dr2, dr2)), SG_M(dr3, dr3));
    const double amj = m[j];
    const double fourhpi2 = fabs(r2in[i]), fourhpj2 = fabs(r2in[j]);
    double gacc, gpot;
    if (r2 >= fmax(fourhpi2, fourhpj2)) {
        const double rinv = SG_D(1.0, __dsqrt_rn(r2));
        const double mrinv1 = SG_M(rinv, amj);
        gacc = SG_M(SG_M(rinv, rinv), mrinv1);
        gpot = -mrinv1;
    } else if (r2 > 0.0) {
        const double rinv = SG_D(1.0, __dsqrt_rn(r2));
        const double mrinv1 = SG_M(rinv, amj);
        near_kernel_f64(nkernel, r2, rinv, amj, __dsqrt_rn(fourhpi2), fourhpi2,
                        __dsqrt_rn(fourhpj2), fourhpj2, mrinv1, SG_M(SG_M(rinv, rinv), mrinv1),
                        gacc, gpot);
    } else {
        gacc = 0.0;
        const double twohpi = __dsqrt_rn(fourhpi2), twohpj = __dsqrt_rn(fourhpj2);
        const double s = SG_A(SG_D(amj, twohpi), SG_D(amj, twohpj));
        const double c = self_c(nkernel);
        if (i == j)
            gpot = r2in[i] > 0.0 ? SG_M(-c, s) : 0.0;
        else
            gpot = r2in[min(i, j)] > 0.0 ? SG_M(SG_M(-0.5, c), s) : 0.0;
    }
    PairOut o;
    o.ax = SG_M(gacc, dr1);
    o.ay = SG_M(gacc, dr2);
    o.az = SG_M(gacc, dr3);
    o.pot = gpot;
    return o;
}

__global__ void __launch_bounds__(NA_NT) k_fp64_noalloc(int n, const double *x, const double *y,
                                                        const double *z, const double *m,
                                                        const double *r2in, int nkernel,
                                                        int nchunks, double *part)
{
    __shared__ double s_x[NA_TJ], s_y[NA_TJ], s_z[NA_TJ], s_m[NA_TJ], s_h[NA_TJ];
    const int i = blockIdx.x * NA_NT + threadIdx.x;
    const int c = blockIdx.y;
    const int j0 = (int)((long long)n * c / nchunks), j1 = (int)((long long)n * (c + 1) / nchunks);
    const bool act = i < n;
    const double xi = act ? x[i] : 1e15, yi = act ? y[i] : 1e15, zi = act ? z[i] : -1e15;
    const double hi2 = act ? fabs(r2in[i]) : 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0, pot = 0.0;
    for (int jt = j0; jt < j1; jt += NA_TJ) {
        const int j = jt + threadIdx.x;
        if (j < j1) {
            s_x[threadIdx.x] = x[j];
            s_y[threadIdx.x] = y[j];
            s_z[threadIdx.x] = z[j];
            s_m[threadIdx.x] = m[j];
            s_h[threadIdx.x] = fabs(r2in[j]);
        }
        __syncthreads();
        const int cnt = min(NA_TJ, j1 - jt);
        for (int k = 0; k < cnt; k++) {
            const double dx = s_x[k] - xi, dy = s_y[k] - yi, dz = s_z[k] - zi;
            const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
            if (r2 >= fmax(hi2, s_h[k])) {
                const double rinv = rsqrt(r2);
                const double mr = s_m[k] * rinv;
                const double mr3 = mr * rinv * rinv;
                ax = fma(mr3, dx, ax);
                ay = fma(mr3, dy, ay);
                az = fma(mr3, dz, az);
                pot -= mr;
            } else if (act) {
                const PairOut o = pair_f64_raw(x, y, z, m, r2in, nkernel, i, jt + k);
                ax += o.ax;
                ay += o.ay;
                az += o.az;
                pot += o.pot;
            }
        }
        __syncthreads();
    }
    if (act) {
        double *p = part + (size_t)c * 4 * n;
        p[i] = ax;
        p[(size_t)n + i] = ay;
        p[2 * (size_t)n + i] = az;
        p[3 * (size_t)n + i] = pot;
    }
}

__global__ void k_merge_noalloc(int n, int nchunks, const double *part, double *ax, double *ay,
                                double *az, double *pot)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < nchunks; c++)
        for (int q = 0; q < 4; q++) s[q] += part[((size_t)c * 4 + q) * n + i];
    ax[i] = s[0];
    ay[i] = s[1];
    az[i] = s[2];
    pot[i] = s[3];
}

}  // namespace sg

using namespace sg;

// Device address of the static scratch, looked up once per device.  Atomic:
// host threads calling on different devices (or racing on the first call of
// one device, which both resolve to the same address) must not race.
static std::atomic<void *> g_noalloc_ptr[64];

extern "C" int sphgrav_forces_fp64_noalloc(int n, const double *x, const double *y,
                                           const double *z, const double *mass,
                                           const double *range2, int nkernel, double *ax,
                                           double *ay, double *az, double *pot, void *stream)
{
    if (n < 0 || nkernel < 0 || nkernel > 2) return SPHGRAV_ERR_INVALID_ARGUMENT;
    if (n > SPHGRAV_NOALLOC_MAX_N) return SPHGRAV_ERR_TOO_LARGE;
    if (n == 0) return SPHGRAV_OK;
    if (!x || !y || !z || !mass || !range2 || !ax || !ay || !az || !pot)
        return SPHGRAV_ERR_INVALID_ARGUMENT;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return SPHGRAV_ERR_NO_DEVICE;
    }
    void *part_p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!part_p) {
        // set-up on this device's first call (host code cannot use the
        // symbol's name as a device address)
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return SPHGRAV_ERR_CUDA;
        }
        g_noalloc_ptr[dev].store(p, std::memory_order_release);
        part_p = p;
    }
    double *part = (double *)part_p;
    // j-chunks: enough blocks to fill the GPU at small n, within the scratch
    const long long per_chunk = 4ll * n;
    int nchunks = (int)std::min<long long>(16, (long long)NA_SCRATCH_DOUBLES / per_chunk);
    nchunks = std::max(1, std::min(nchunks, (n + 2047) / 2048));
    cudaStream_t st = (cudaStream_t)stream;
    dim3 grid((n + NA_NT - 1) / NA_NT, nchunks);
    k_fp64_noalloc<<<grid, NA_NT, 0, st>>>(n, x, y, z, mass, range2, nkernel, nchunks, part);
    k_merge_noalloc<<<(n + 255) / 256, 256, 0, st>>>(n, nchunks, part, ax, ay, az, pot);
    g_launches += 2;
    if (cudaGetLastError() != cudaSuccess) return SPHGRAV_ERR_CUDA;
    return SPHGRAV_OK;
}
