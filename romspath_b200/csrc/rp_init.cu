// rp_init.cu -- the initialisation lookups: LL2ij of every particle on the
// device (interpolation_module.f90:110-268) and InitGrid's nest maps
// (grid_module.f90:437-481) on the host.  Compiled without FMA contraction
// so that the fractional indices match the oracle's bit for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "romspath_gpu.h"
#include "rp_geo.cuh"
#include "rp_internal.h"

namespace rp {

constexpr int kInitBlock = 128;

// One thread per particle; the first inbox walks the whole grid boundary,
// which every thread of a warp reads at the same address.
__global__ void __launch_bounds__(kInitBlock) k_ll2ij(const double* __restrict__ lon, const double* __restrict__ lat,
                                                     const double* __restrict__ angle, int nx, int ny, int spherical,
                                                     const double* __restrict__ inlon,
                                                     const double* __restrict__ inlat, int64_t n,
                                                     double* __restrict__ ip, double* __restrict__ jp) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        double a, b;
        rp_ll2ij_one(lon, lat, angle, nx, ny, spherical, inlon[k], inlat[k], a, b);
        ip[k] = a;
        jp[k] = b;
    }
}

cudaError_t launch_ll2ij(const double* lon, const double* lat, const double* angle, int nx, int ny, int spherical,
                         const double* inlon, const double* inlat, int64_t n, double* ip, double* jp, int num_sms,
                         cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int64_t blocks = (n + kInitBlock - 1) / kInitBlock;
    const int64_t cap = (int64_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_ll2ij<<<(unsigned)blocks, kInitBlock, 0, s>>>(lon, lat, angle, nx, ny, spherical, inlon, inlat, n, ip, jp);
    return cudaGetLastError();
}

}  // namespace rp

namespace {

// Fortran .EQ. on two doubles: equal values, +0 equal to -0, NaN never
// equal; the key is the value's bits with -0 folded onto +0.
uint64_t eq_key(double v) {
    if (v == 0.0) v = 0.0;
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}

struct PairKey {
    uint64_t a, b;
    bool operator==(const PairKey& o) const { return a == o.a && b == o.b; }
};
struct PairHash {
    size_t operator()(const PairKey& k) const { return (size_t)(k.a * 0x9E3779B97F4A7C15ull ^ (k.b + (k.a >> 7))); }
};

}  // namespace

extern "C" {

int rp_nest_maps(int32_t ngrid, const int32_t* xi_rho, const int32_t* eta_rho, const double* const* lon_rho,
                 const double* const* lat_rho, const double* refine, double* scl, double* off) {
    if (ngrid < 1 || ngrid > RP_MAXNGRID || !xi_rho || !eta_rho || !lon_rho || !lat_rho || !scl || !off)
        return RP_ERR_ARG;
    if (ngrid > 1 && !refine) return RP_ERR_ARG;
    for (int g = 0; g < ngrid; g++)
        if (xi_rho[g] < 1 || eta_rho[g] < 1 || !lon_rho[g] || !lat_rho[g]) return RP_ERR_ARG;
    double grefine[RP_MAXNGRID][RP_MAXNGRID];
    for (int a = 0; a < ngrid; a++)                        // grid_module.f90:437-450
        for (int b = 0; b < ngrid; b++) {
            grefine[a][b] = 1.0;
            const int dng = a > b ? a - b : b - a;
            for (int r = 1; r <= dng; r++) grefine[a][b] = refine[dng - 1] * grefine[a][b];
        }
    for (int k = 0; k < ngrid * 2 * ngrid; k++) {
        scl[k] = 1.0;
        off[k] = 0.0;
    }
    auto S = [&](int ng, int c, int i) -> double& { return scl[((size_t)ng * 2 + c) * ngrid + i]; };
    auto O = [&](int ng, int c, int i) -> double& { return off[((size_t)ng * 2 + c) * ngrid + i]; };
    // first (ii, jj) of each coincident (lon, lat) in grid B, ii slowest
    std::vector<std::unordered_map<PairKey, std::pair<int, int>, PairHash>> first(ngrid);
    for (int g = 0; g < ngrid; g++) {
        auto& m = first[g];
        m.reserve((size_t)xi_rho[g] * eta_rho[g]);
        for (int ii = 1; ii <= xi_rho[g]; ii++)
            for (int jj = 1; jj <= eta_rho[g]; jj++) {
                const size_t o = (size_t)(jj - 1) * xi_rho[g] + (ii - 1);
                const double lo = lon_rho[g][o], la = lat_rho[g][o];
                if (lo != lo || la != la) continue;
                m.emplace(PairKey{eq_key(lo), eq_key(la)}, std::make_pair(ii, jj));
            }
    }
    for (int ng2 = 0; ng2 < ngrid; ng2++) {                // 454-481, the reference's search order
        for (int ng = 0; ng < ngrid; ng++) {
            const auto& m = first[ng2];
            // no coincident point: the indices past the loops' ends
            int i = xi_rho[ng] + 1, j = eta_rho[ng] + 1, ii = xi_rho[ng2] + 1, jj = eta_rho[ng2] + 1;
            bool hit = false;
            for (int a = 1; a <= xi_rho[ng] && !hit; a++)
                for (int b = 1; b <= eta_rho[ng] && !hit; b++) {
                    const size_t o = (size_t)(b - 1) * xi_rho[ng] + (a - 1);
                    const double lo = lon_rho[ng][o], la = lat_rho[ng][o];
                    if (lo != lo || la != la) continue;
                    auto it = m.find(PairKey{eq_key(lo), eq_key(la)});
                    if (it != m.end()) {
                        hit = true;
                        i = a; j = b; ii = it->second.first; jj = it->second.second;
                    }
                }
            for (int c = 0; c < 2; c++) {
                S(ng, c, ng2) = 1.0 / grefine[ng][ng2];
                S(ng2, c, ng) = grefine[ng2][ng];
            }
            O(ng, 0, ng2) = (double)ii - S(ng, 0, ng2) * (double)i;
            O(ng, 1, ng2) = (double)jj - S(ng, 1, ng2) * (double)j;
            O(ng2, 0, ng) = (double)i - S(ng2, 0, ng) * (double)ii;
            O(ng2, 1, ng) = (double)j - S(ng2, 1, ng) * (double)jj;
        }
    }
    return RP_OK;
}

}  // extern "C"
