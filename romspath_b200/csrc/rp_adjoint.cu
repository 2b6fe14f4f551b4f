// rp_adjoint.cu -- kernels of the adjoint pair (rp_forward / rp_backward),
// the tangent-linear reference and the replay used by finite differences.
// All of them run the one generic step of rp_adjoint.cuh; compiled without
// FMA contraction so that the double and the dual instantiations take the
// same values.
#include <cuda_runtime.h>

#include "rp_internal.h"
#include "rp_adjoint.cuh"

namespace rp {

constexpr int kAdjBlock = 128;

__device__ __forceinline__ void adj_load(const AdjStateDev& s, int64_t n, double& x, double& y, double& z,
                                         AdjAux& a) {
    x = s.x[n];
    y = s.y[n];
    z = s.z[n];
    a.age = s.age[n];
    a.status = s.status[n];
    a.gid = s.gid[n];
    a.isin = s.isin[n];
}

__device__ __forceinline__ void adj_store_aux(const AdjStateDev& s, int64_t n, const AdjAux& a) {
    s.age[n] = a.age;
    s.status[n] = a.status;
    s.gid[n] = a.gid;
    s.isin[n] = a.isin;
}

// one step of the model in doubles on state s; find: search p and record
// it in prec[n], else use prec[n]
template <int NPMAX>
__global__ void __launch_bounds__(kAdjBlock) k_adj_step(const __grid_constant__ RpStepArgs A,
                                                         const __grid_constant__ AdjFrames F, AdjStateDev s,
                                                         double* __restrict__ prec, int find, double kappa) {
    double buf[kAdjArrays * (NPMAX + 1)];
    const AFit<double, NPMAX> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride) {
        double x, y, z;
        AdjAux a;
        adj_load(s, n, x, y, z, a);
        double p = find ? 0.0 : prec[n];
        uint32_t fl = 0;
        a_step<double, NPMAX>(A, F, A.p.dob[n], A.p.pid[n], x, y, z, a, kappa, find != 0, p, fl, w);
        if (find) prec[n] = p;
        s.x[n] = x;
        s.y[n] = y;
        s.z[n] = z;
        adj_store_aux(s, n, a);
    }
}

// one step in dual numbers carrying d/d(x0, y0, z0, kappa): tangent-linear
// propagation; t holds the 12 derivatives of (x, y, z) per particle
template <int NPMAX>
__global__ void __launch_bounds__(kAdjBlock) k_adj_tangent(const __grid_constant__ RpStepArgs A,
                                                            const __grid_constant__ AdjFrames F, AdjStateDev s,
                                                            double* __restrict__ t, const double* __restrict__ prec,
                                                            double kappa) {
    using D = Dual<4>;
    D buf[kAdjArrays * (NPMAX + 1)];
    const AFit<D, NPMAX> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride) {
        double x, y, z;
        AdjAux a;
        adj_load(s, n, x, y, z, a);
        D X(x), Y(y), Z(z), K(kappa);
        double* tn = t + n * 12;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            X.d[q] = tn[q];
            Y.d[q] = tn[4 + q];
            Z.d[q] = tn[8 + q];
        }
        K.d[3] = 1.0;
        double p = prec[n];
        uint32_t fl = 0;
        a_step<D, NPMAX>(A, F, A.p.dob[n], A.p.pid[n], X, Y, Z, a, K, false, p, fl, w);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            tn[q] = X.d[q];
            tn[4 + q] = Y.d[q];
            tn[8 + q] = Z.d[q];
        }
        s.x[n] = X.v;
        s.y[n] = Y.v;
        s.z[n] = Z.v;
        adj_store_aux(s, n, a);
    }
}

// one reverse step: from the step's starting state s (read only), the
// step's Jacobian by dual numbers seeded on (x, y, z, kappa); then
// lambda <- J^T lambda for (x, y, z) and kbar += lambda . d(x,y,z)/dkappa
template <int NPMAX>
__global__ void __launch_bounds__(kAdjBlock) k_adj_reverse(const __grid_constant__ RpStepArgs A,
                                                            const __grid_constant__ AdjFrames F, AdjStateDev s,
                                                            const double* __restrict__ prec, double kappa,
                                                            double* __restrict__ lx, double* __restrict__ ly,
                                                            double* __restrict__ lz, double* __restrict__ kbar) {
    using D = Dual<4>;
    D buf[kAdjArrays * (NPMAX + 1)];
    const AFit<D, NPMAX> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride) {
        double x, y, z;
        AdjAux a;
        adj_load(s, n, x, y, z, a);
        D X(x), Y(y), Z(z), K(kappa);
        X.d[0] = 1.0;
        Y.d[1] = 1.0;
        Z.d[2] = 1.0;
        K.d[3] = 1.0;
        double p = prec[n];
        uint32_t fl = 0;
        a_step<D, NPMAX>(A, F, A.p.dob[n], A.p.pid[n], X, Y, Z, a, K, false, p, fl, w);
        const double bx = lx[n], by = ly[n], bz = lz[n];
        lx[n] = bx * X.d[0] + by * Y.d[0] + bz * Z.d[0];
        ly[n] = bx * X.d[1] + by * Y.d[1] + bz * Z.d[1];
        lz[n] = bx * X.d[2] + by * Y.d[2] + bz * Z.d[2];
        kbar[n] += bx * X.d[3] + by * Y.d[3] + bz * Z.d[3];
    }
}

template <class K>
static int64_t adj_grid(K kernel, int64_t n, int num_sms) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kAdjBlock, 0) != cudaSuccess || occ < 1) occ = 1;
    int64_t b = (int64_t)num_sms * occ;
    const int64_t need = (n + kAdjBlock - 1) / kAdjBlock;
    if (need < b) b = need;
    return b < 1 ? 1 : b;
}

template <int NPMAX>
static cudaError_t adj_launch_t(int kind, const RpStepArgs& A, const AdjFrames& F, const AdjStateDev& s,
                                double* prec, int find, double kappa, double* t, double* lx, double* ly, double* lz,
                                double* kbar, cudaStream_t st, int num_sms) {
    if (kind == 0) {
        k_adj_step<NPMAX><<<(unsigned)adj_grid(k_adj_step<NPMAX>, A.p.n, num_sms), kAdjBlock, 0, st>>>(A, F, s, prec,
                                                                                                      find, kappa);
    } else if (kind == 1) {
        k_adj_tangent<NPMAX><<<(unsigned)adj_grid(k_adj_tangent<NPMAX>, A.p.n, num_sms), kAdjBlock, 0, st>>>(
            A, F, s, t, prec, kappa);
    } else {
        k_adj_reverse<NPMAX><<<(unsigned)adj_grid(k_adj_reverse<NPMAX>, A.p.n, num_sms), kAdjBlock, 0, st>>>(
            A, F, s, prec, kappa, lx, ly, lz, kbar);
    }
    return cudaGetLastError();
}

cudaError_t launch_adj(int kind, const RpStepArgs& A, const AdjFrames& F, const AdjStateDev& s, double* prec, int find,
                       double kappa, double* t, double* lx, double* ly, double* lz, double* kbar, int npmax,
                       cudaStream_t st, int num_sms) {
    if (A.p.n <= 0) return cudaSuccess;
    if (npmax <= 88) return adj_launch_t<88>(kind, A, F, s, prec, find, kappa, t, lx, ly, lz, kbar, st, num_sms);
    if (npmax <= 128) return adj_launch_t<128>(kind, A, F, s, prec, find, kappa, t, lx, ly, lz, kbar, st, num_sms);
    return adj_launch_t<144>(kind, A, F, s, prec, find, kappa, t, lx, ly, lz, kbar, st, num_sms);
}

// Fortran-ordered field (+ Stokes term, summed in FP64) -> [j][i][k] FP64
template <typename S>
__global__ void k_adj_store(const S* __restrict__ src, const S* __restrict__ add, double* __restrict__ dst, int ni,
                            int nj, int nk, int64_t e0, int64_t count) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int64_t e = e0 + t;
    const int64_t plane = (int64_t)ni * nj;
    const int k = (int)(e / plane);
    const int64_t r = e - (int64_t)k * plane;
    const int j = (int)(r / ni);
    const int i = (int)(r - (int64_t)j * ni);
    double v = (double)src[t];
    if (add) v = v + (double)add[t];
    dst[((int64_t)j * ni + i) * nk + k] = v;
}

cudaError_t launch_adj_store(const double* src, const double* add, double* dst, int ni, int nj, int nk, int64_t e0,
                             int64_t count, cudaStream_t s) {
    const unsigned nb = (unsigned)((count + 255) / 256);
    if (nb == 0) return cudaSuccess;
    k_adj_store<double><<<nb, 256, 0, s>>>(src, add, dst, ni, nj, nk, e0, count);
    return cudaGetLastError();
}

// initial tangent: d(x, y, z)/d(x0, y0, z0, kappa) = [I 0]
__global__ void k_adj_tangent_init(double* t, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* tn = t + i * 12;
#pragma unroll
    for (int q = 0; q < 12; q++) tn[q] = 0.0;
    tn[0] = 1.0;
    tn[5] = 1.0;
    tn[10] = 1.0;
}

cudaError_t launch_adj_tangent_init(double* t, int64_t n, cudaStream_t s) {
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (nb == 0) return cudaSuccess;
    k_adj_tangent_init<<<nb, 256, 0, s>>>(t, n);
    return cudaGetLastError();
}

}  // namespace rp
