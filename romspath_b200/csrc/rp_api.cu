// rp_api.cu -- the C ABI (include/romspath_gpu.h): context, HBM layout,
// frame ring, particle state and step launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "romspath_gpu.h"
#include "rp_internal.h"

namespace {

constexpr int64_t kChunkElems = 4 << 20;     // staging chunk (elements)
using rp::kMaxNp;

struct GridBuf {
    int nx = 0, ny = 0, N = 0, vtransform = 2;
    double hc = 0.0;
    double *h = nullptr, *pm = nullptr, *pn = nullptr;
    double *sr = nullptr, *csr = nullptr, *sw = nullptr, *csw = nullptr;
    float2 *scs_r = nullptr, *scs_w = nullptr;   // the same in FP32 pairs (s, Cs)
    float2* hm = nullptr;                        // (h, mask_rho) in FP32
    uint8_t *mrho = nullptr, *mu = nullptr, *mv = nullptr;
    void *zeta = nullptr, *u = nullptr, *v = nullptr, *w = nullptr, *aks = nullptr;
    void *salt = nullptr, *temp = nullptr, *bustr = nullptr, *bvstr = nullptr;  // diagnostics only
    double *lon = nullptr, *lat = nullptr;     // lon_rho, lat_rho (output records, LL2ij)
    double* angle = nullptr;                   // GRIDS(ng)%angle (LL2ij, spherical grids)
    int spherical = -1;                        // GRIDS(ng)%spherical (-1: not set)
    uint8_t *wd_rho = nullptr, *wd_u = nullptr, *wd_v = nullptr;  // WETDRY masks, [j][i][slot4]
    void *turbaccel = nullptr, *turbvort = nullptr;      // behave's fields (Process_VA)
    void *waveaccelu = nullptr, *waveaccelv = nullptr;   // (Process_WA)
    float *qs_u = nullptr, *qs_v = nullptr, *qs_w = nullptr, *qs_aks = nullptr;  // mixed form: [k][slot4]
    double scl[RP_MAXNGRID][2] = {}, off[RP_MAXNGRID][2] = {};
    int map[3] = {-1, -1, -1};                 // logical slot 1..3 -> physical 0..3
    bool slot_loaded[RP_SLOTS] = {false, false, false, false};
    bool free_recorded[RP_SLOTS] = {false, false, false, false};
    cudaEvent_t slot_free[RP_SLOTS] = {};      // last reader of the physical slot done
    cudaEvent_t slot_ready[RP_SLOTS] = {};     // upload into the physical slot done
};

}  // namespace

struct rp_ctx {
    rp_params prm{};
    int ngrid = 0;
    int device = 0;
    int num_sms = 148;
    int elem = 8;                              // bytes per stored field value (FP64/FP32 forms)
    bool mixed = false;                        // RP_FIELD_MIXED or RP_FIELD_MIXED_I16
    bool i16 = false;                          // RP_FIELD_MIXED_I16: int16 fixed point instead of FP16
    int npmax = 0;
    GridBuf g[RP_MAXNGRID];
    // particle state
    int64_t cap = 0, n = 0;
    double *x = nullptr, *y = nullptr, *z = nullptr, *age = nullptr, *dob = nullptr, *status = nullptr;
    double *wd = nullptr, *zeta = nullptr, *bath = nullptr;
    int32_t* gid = nullptr;
    int8_t* isin = nullptr;
    uint32_t *pid = nullptr, *flags = nullptr;
    double* turbv = nullptr;                   // scratch, 12 B per particle: the re-sort's gathers; the mixed
                                               // form's VTurb displacement, tdepth and ZBehav (3 floats)
    // diagnostics (RP_DIAG_* bits of reserved[3]); null when off
    int diag = 0;
    double *d_salt = nullptr, *d_temp = nullptr, *d_mean_salt = nullptr, *d_mean_temp = nullptr;
    double *d_hob = nullptr, *d_bustr = nullptr, *d_bvstr = nullptr;
    double* outbuf = nullptr;                  // packed output record: kOutCols x cap doubles
    bool wetdry = false;                       // WETDRY (reserved[4])
    // behave: parameters (rp_set_behavior), its outputs per particle
    bool beh_set = false;
    RpBehaviorDev beh{};
    double *b_acc = nullptr, *b_vort = nullptr, *b_behavew = nullptr, *b_ssf = nullptr;
    uint8_t* wd_stage = nullptr;               // one mask of a frame on its way into the ring
    // mixed form: compensated FP32 positions, spline warm start, and the
    // FP32 staging field plus per-level maxima of the FP16 quantisation
    float *x32 = nullptr, *y32 = nullptr, *z32 = nullptr, *cx = nullptr, *cy = nullptr, *cz = nullptr;
    double* qwarm = nullptr;
    double* gwarm = nullptr;
    float* qwarm2 = nullptr;
    float* ftmp = nullptr;
    uint32_t* qmax = nullptr;
    double* tmp_gid = nullptr;                 // host-facing conversions
    int32_t* tmp_isin = nullptr;
    // staging
    void* pin[2] = {nullptr, nullptr};         // pinned, 2 x (2 arrays x chunk x 8 B)
    void* dstage[2] = {nullptr, nullptr};      // device, same shape
    cudaEvent_t pin_done[2] = {};
    bool pin_used[2] = {false, false};
    int pin_next = 0;
    cudaStream_t s_comp = nullptr, s_copy = nullptr;
    cudaStream_t s_out = nullptr;              // read-back of asynchronous output records
    cudaEvent_t ev_packed = nullptr, ev_out_done = nullptr;
    cudaEvent_t ev_na_in = nullptr, ev_na_out = nullptr;   // rp_step_noalloc: caller stream <-> compute stream
    bool out_pending = false;                  // an asynchronous record's copies may be in flight
    // noise hook
    double* hook = nullptr;
    int64_t hook_steps = 0, hook_pos = 0;
    int ndraw = 0;
    uint64_t step_index = 0;
    uint32_t pid_base = 0;
    // timing
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    int last_kernels = 0;
    bool direct_pending = false;               // an upload read the caller's pinned arrays by DMA
    cudaGraphExec_t gexec = nullptr;           // rp_step_n's graph of one call's launches
    // re-sorting by cell: every `resort` internal steps (0: never)
    int resort = 0;
    int64_t since_sort = 0;
    bool permuted = false;                     // columns not in the caller's order
    uint32_t state_base = 0;                   // id base of the current particle set
    rp::SortBufs sb;
    // adjoint pair: frame store, step table, checkpoints, recorded smoothing
    // parameters and the backward sweep's buffers
    struct Adj {
        int nframes = 0;
        double* fst[RP_MAXNGRID][5] = {};      // [frame][j][i][k] per field
        size_t fsize[RP_MAXNGRID][5] = {};     // values per frame
        std::vector<rp_adj_step> steps;
        int ckpt = 0;
        int64_t n = 0;                         // particles of the recorded run
        double kappa = 1.0;
        double* ck = nullptr;                  // checkpoints: (nsteps/ckpt + 1) state blocks
        double* prec = nullptr;                // recorded p: nsteps x n
        double* seg = nullptr;                 // one segment of step-start states: ckpt blocks
        double* work = nullptr;                // working state block
        double *lx = nullptr, *ly = nullptr, *lz = nullptr, *kbar = nullptr, *tan = nullptr;
        size_t cap_steps = 0;
    } adj;
    int64_t launches = 0;
    // smoothing-spline fits and chol1d passes counted by the step kernels
    unsigned long long* d_spl = nullptr;
    bool spl_on = false;
    std::string err;
};

namespace {

int fail(rp_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(ctx, RP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename P>
cudaError_t dalloc(P** p, size_t bytes) {
    return cudaMalloc((void**)p, bytes ? bytes : 1);
}

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// host -> device through the pinned staging halves, on stream s (direct
// when the caller's buffer is already page-locked)
int h2d(rp_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes && is_pinned(src)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return RP_OK;
    }
    const size_t chunk = (size_t)kChunkElems * 8 * 2;
    size_t done = 0;
    while (done < bytes) {
        const size_t nb = std::min(chunk, bytes - done);
        const int h = ctx->pin_next;
        ctx->pin_next ^= 1;
        if (ctx->pin_used[h]) CK(cudaEventSynchronize(ctx->pin_done[h]));
        std::memcpy(ctx->pin[h], (const char*)src + done, nb);
        CK(cudaMemcpyAsync((char*)dst + done, ctx->pin[h], nb, cudaMemcpyHostToDevice, s));
        CK(cudaEventRecord(ctx->pin_done[h], s));
        ctx->pin_used[h] = true;
        done += nb;
    }
    return RP_OK;
}

// device -> host through the pinned staging halves (synchronous; direct
// when the caller's buffer is already page-locked)
int d2h(rp_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes && is_pinned(dst)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return RP_OK;
    }
    const size_t chunk = (size_t)kChunkElems * 8 * 2;
    size_t done = 0;
    while (done < bytes) {
        const size_t nb = std::min(chunk, bytes - done);
        const int h = ctx->pin_next;
        ctx->pin_next ^= 1;
        if (ctx->pin_used[h]) CK(cudaEventSynchronize(ctx->pin_done[h]));
        CK(cudaMemcpyAsync(ctx->pin[h], (const char*)src + done, nb, cudaMemcpyDeviceToHost, s));
        CK(cudaEventRecord(ctx->pin_done[h], s));
        CK(cudaEventSynchronize(ctx->pin_done[h]));
        ctx->pin_used[h] = false;
        std::memcpy((char*)dst + done, ctx->pin[h], nb);
        done += nb;
    }
    return RP_OK;
}

RpParticlesDev particles_dev(const rp_ctx* c) {
    RpParticlesDev P;
    P.n = c->n;
    P.x = c->x; P.y = c->y; P.z = c->z; P.age = c->age; P.dob = c->dob; P.status = c->status;
    P.wd = c->wd; P.zeta = c->zeta; P.bath = c->bath;
    P.gid = c->gid; P.isin = c->isin; P.pid = c->pid; P.flags = c->flags;
    P.x32 = c->x32; P.y32 = c->y32; P.z32 = c->z32; P.cx = c->cx; P.cy = c->cy; P.cz = c->cz;
    P.qwarm = c->qwarm; P.gwarm = c->gwarm; P.qwarm2 = c->qwarm2;
    P.salt = c->d_salt; P.temp = c->d_temp; P.mean_salt = c->d_mean_salt; P.mean_temp = c->d_mean_temp;
    P.hob = c->d_hob; P.bustr = c->d_bustr; P.bvstr = c->d_bvstr;
    P.acc = c->b_acc; P.vort = c->b_vort; P.behavew = c->b_behavew; P.ssf = c->b_ssf;
    return P;
}

void fill_grids(const rp_ctx* c, RpStepArgs& A, int tb, int tc, int tf) {
    for (int k = 0; k < c->ngrid; k++) {
        const GridBuf& G = c->g[k];
        RpGridDev& d = A.g[k];
        d.nx = G.nx; d.ny = G.ny; d.N = G.N; d.vtransform = G.vtransform; d.hc = G.hc;
        d.h = G.h; d.pm = G.pm; d.pn = G.pn;
        d.mrho = G.mrho; d.mu = G.mu; d.mv = G.mv;
        d.sr = G.sr; d.csr = G.csr; d.sw = G.sw; d.csw = G.csw;
        d.scs_r = G.scs_r; d.scs_w = G.scs_w; d.hm = G.hm;
        d.zeta = G.zeta; d.u = G.u; d.v = G.v; d.w = G.w; d.aks = G.aks;
        d.salt = G.salt; d.temp = G.temp; d.bustr = G.bustr; d.bvstr = G.bvstr;
        d.lon = G.lon; d.lat = G.lat;
        d.wd_rho = G.wd_rho; d.wd_u = G.wd_u; d.wd_v = G.wd_v;
        d.turbaccel = G.turbaccel; d.turbvort = G.turbvort; d.waveaccelu = G.waveaccelu; d.waveaccelv = G.waveaccelv;
        d.qs_u = G.qs_u; d.qs_v = G.qs_v; d.qs_w = G.qs_w; d.qs_aks = G.qs_aks;
        for (int i = 0; i < RP_MAXNGRID; i++)
            for (int q = 0; q < 2; q++) { d.scl[i][q] = G.scl[i][q]; d.off[i][q] = G.off[i][q]; }
        d.sb = (tb >= 1 && tb <= 3) ? G.map[tb - 1] : 0;
        d.sc = (tc >= 1 && tc <= 3) ? G.map[tc - 1] : 0;
        d.sf = (tf >= 1 && tf <= 3) ? G.map[tf - 1] : 0;
    }
}

void fill_params(const rp_ctx* c, RpStepArgs& A) {
    const rp_params& p = c->prm;
    A.ngrid = c->ngrid;
    A.idt = p.idt; A.scheme = p.scheme; A.nsb = p.nsb;
    A.vturb_on = p.vturb_on; A.hturb_on = p.hturb_on; A.oob = p.open_ocean_boundary;
    A.loop = p.idt / (int)p.deltat;
    A.grid_cap = p.reserved[2] > 0 ? p.reserved[2] : 0;
    A.spline_max_iter = p.spline_max_iter > 0 ? p.spline_max_iter : 100;
    A.diag = c->diag;
    A.wetdry = c->wetdry ? 1 : 0;
    A.beh = c->beh;
    A.vertdist = p.vertdist; A.serr = p.serr; A.smth = p.smth; A.sub = p.sub;
    A.deltat = p.deltat; A.aksback = p.aksback;
    for (int i = 0; i < RP_MAXNGRID; i++) A.khturb[i] = p.constant_hturb[i];
    A.seed = p.seed;
    A.ndraw = c->ndraw;
    A.pid_base = c->pid_base;
    A.spl = c->spl_on ? c->d_spl : nullptr;
    A.p = particles_dev(c);
}

// polintd node terms (interpolation_module.f90:72-109) for nodes xa, point x
RpPolint polint_consts(const double xa[3], double x) {
    RpPolint P;
    int ns = 0;
    double dif = std::fabs(x - xa[0]);
    for (int i = 0; i < 3; i++) {
        const double dift = std::fabs(x - xa[i]);
        if (dift < dif) { ns = i; dif = dift; }
    }
    P.ns = ns;
    P.d1 = xa[1] - x;
    P.e12 = xa[1] - xa[2];
    P.e01 = xa[0] - xa[1];
    P.e02 = xa[0] - xa[2];
    P.dns = xa[ns] - x;
    P.b = (ns == 2) ? (xa[2] - x) : (xa[0] - x);
    P.re12 = 1.0 / P.e12;
    P.re01 = 1.0 / P.e01;
    P.re02 = 1.0 / P.e02;
    return P;
}

// The mixed form's per-step slot data of every grid: A.lw summed by the
// physical slot each of t_b, t_c, t_f sits in, and masks of the live FP32
// slots (the spare one is read with every float4 and must meet a weight of
// 0 and no bits of its own: an upload may be filling it)
void slot_weights(RpStepArgs& A, int ngrid) {
    for (int k = 0; k < ngrid; k++) {
        RpGridDev& d = A.g[k];
        const int sl[3] = {d.sb, d.sc, d.sf};
        for (int which = 0; which < 2; which++) {
            float w[4] = {0.f, 0.f, 0.f, 0.f};
            for (int q = 0; q < 3; q++) w[sl[q]] += A.lw[which][q];
            d.w4[which] = make_float4(w[0], w[1], w[2], w[3]);
        }
        uint32_t live[4];
        for (int s = 0; s < 4; s++) live[s] = (sl[0] == s || sl[1] == s || sl[2] == s) ? 0xffffffffu : 0u;
        d.m32 = make_uint4(live[0], live[1], live[2], live[3]);
    }
}

// polintd's interpolant at x as Lagrange weights of its three values (the
// mixed form folds them into the gathers): [0] for (b, c, f), [1] for the
// u/v/w values, which at ets == 1 are (b, b, c) (advection_module.f90:277-287)
void lagrange_weights(const double xa[3], double x, int ets, float lw[2][3]) {
    const double a0 = (x - xa[1]) * (x - xa[2]) / ((xa[0] - xa[1]) * (xa[0] - xa[2]));
    const double a1 = (x - xa[0]) * (x - xa[2]) / ((xa[1] - xa[0]) * (xa[1] - xa[2]));
    const double a2 = (x - xa[0]) * (x - xa[1]) / ((xa[2] - xa[0]) * (xa[2] - xa[1]));
    lw[0][0] = (float)a0; lw[0][1] = (float)a1; lw[0][2] = (float)a2;
    if (ets == 1) {
        lw[1][0] = (float)(a0 + a1); lw[1][1] = (float)a2; lw[1][2] = 0.f;
    } else {
        lw[1][0] = lw[0][0]; lw[1][1] = lw[0][1]; lw[1][2] = lw[0][2];
    }
}

void free_ctx(rp_ctx* c) {
    if (!c) return;
    for (int k = 0; k < RP_MAXNGRID; k++) {
        GridBuf& G = c->g[k];
        void* ptrs[] = {G.h, G.pm, G.pn, G.sr, G.csr, G.sw, G.csw, G.scs_r, G.scs_w, G.hm, G.mrho, G.mu, G.mv,
                        G.zeta, G.u, G.v, G.w, G.aks, G.qs_u, G.qs_v, G.qs_w, G.qs_aks,
                        G.salt, G.temp, G.bustr, G.bvstr, G.lon, G.lat, G.wd_rho, G.wd_u, G.wd_v,
                        G.turbaccel, G.turbvort, G.waveaccelu, G.waveaccelv, G.angle};
        for (void* p : ptrs) if (p) cudaFree(p);
        for (int s = 0; s < RP_SLOTS; s++) {
            if (G.slot_free[s]) cudaEventDestroy(G.slot_free[s]);
            if (G.slot_ready[s]) cudaEventDestroy(G.slot_ready[s]);
        }
    }
    void* ptrs[] = {c->x, c->y, c->z, c->age, c->dob, c->status, c->wd, c->zeta, c->bath,
                    c->gid, c->isin, c->pid, c->flags, c->tmp_gid, c->tmp_isin, c->hook, c->turbv,
                    c->dstage[0], c->dstage[1], c->x32, c->y32, c->z32, c->cx, c->cy, c->cz, c->qwarm, c->gwarm, c->qwarm2,
                    c->ftmp, c->qmax, c->sb.keys, c->sb.hist, c->sb.sums, c->sb.perm, c->sb.gbase,
                    c->adj.ck, c->adj.prec, c->adj.seg, c->adj.work, c->adj.lx, c->adj.ly, c->adj.lz,
                    c->adj.kbar, c->adj.tan, c->d_salt, c->d_temp, c->d_mean_salt, c->d_mean_temp,
                    c->d_hob, c->d_bustr, c->d_bvstr, c->outbuf, c->wd_stage, c->b_acc, c->b_vort,
                    c->b_behavew, c->b_ssf, c->d_spl};
    for (int g = 0; g < RP_MAXNGRID; g++)
        for (int f = 0; f < 5; f++)
            if (c->adj.fst[g][f]) cudaFree(c->adj.fst[g][f]);
    for (void* p : ptrs) if (p) cudaFree(p);
    for (int h = 0; h < 2; h++) {
        if (c->pin[h]) cudaFreeHost(c->pin[h]);
        if (c->pin_done[h]) cudaEventDestroy(c->pin_done[h]);
    }
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->s_comp) cudaStreamDestroy(c->s_comp);
    if (c->s_copy) cudaStreamDestroy(c->s_copy);
    if (c->s_out) cudaStreamDestroy(c->s_out);
    if (c->ev_packed) cudaEventDestroy(c->ev_packed);
    if (c->ev_na_in) cudaEventDestroy(c->ev_na_in);
    if (c->ev_na_out) cudaEventDestroy(c->ev_na_out);
    if (c->ev_out_done) cudaEventDestroy(c->ev_out_done);
    delete c;
}

// One field of a frame into physical slot `phys`.  FP64/FP32 forms (and the
// FP32 zeta of the mixed form, `f32` set) convert each staged chunk straight
// into the slot; the mixed form's u, v, w, AKs (`qs` non-null) are staged
// whole as FP32, then quantised to FP16 with per-level scales.
template <typename S>
int upload_field(rp_ctx* ctx, const S* src, const S* add, void* dst, int ni, int nj, int nk, int phys,
                 bool f32 = false, float* qs = nullptr) {
    const int64_t total = (int64_t)ni * nj * nk;
    const int dst_f32 = (ctx->elem == 4 || f32);
    const int src_f32 = (sizeof(S) == 4);
    // a page-locked source is copied by DMA straight into the device
    // staging (the call then waits for the copies before returning, since
    // the caller may reuse its arrays); otherwise through our pinned halves
    const bool direct = is_pinned(src) && (!add || is_pinned(add));
    if (direct) ctx->direct_pending = true;
    for (int64_t e0 = 0; e0 < total; e0 += kChunkElems) {
        const int64_t cnt = std::min<int64_t>(kChunkElems, total - e0);
        const size_t nb = (size_t)cnt * sizeof(S);
        const int h = ctx->pin_next;
        ctx->pin_next ^= 1;
        if (ctx->pin_used[h]) CK(cudaEventSynchronize(ctx->pin_done[h]));
        char* pin = (char*)ctx->pin[h];
        char* dst_stage = (char*)ctx->dstage[h];
        const char* from = direct ? (const char*)(src + e0) : pin;
        const char* from_add = direct ? (const char*)(add ? add + e0 : nullptr) : pin + (size_t)kChunkElems * 8;
        if (!direct) {
            std::memcpy(pin, src + e0, nb);
            if (add) std::memcpy(pin + (size_t)kChunkElems * 8, add + e0, nb);
        }
        CK(cudaMemcpyAsync(dst_stage, from, nb, cudaMemcpyHostToDevice, ctx->s_copy));
        if (add)
            CK(cudaMemcpyAsync(dst_stage + (size_t)kChunkElems * 8, from_add, nb, cudaMemcpyHostToDevice,
                               ctx->s_copy));
        if (qs)
            CK(rp::launch_stage_f32(src_f32, dst_stage, add ? dst_stage + (size_t)kChunkElems * 8 : nullptr,
                                    ctx->ftmp, e0, cnt, ctx->s_copy));
        else
            CK(rp::launch_convert(src_f32, dst_f32, dst_stage, add ? dst_stage + (size_t)kChunkElems * 8 : nullptr,
                                  dst, ni, nj, nk, phys, e0, cnt, ctx->s_copy));
        ctx->launches++;
        CK(cudaEventRecord(ctx->pin_done[h], ctx->s_copy));
        ctx->pin_used[h] = true;
    }
    if (qs) {
        CK(rp::launch_quantize(ctx->ftmp, ctx->qmax, qs, dst, ni, nj, nk, phys, ctx->i16, ctx->num_sms, ctx->s_copy));
        ctx->launches += 2;
    }
    return RP_OK;
}

// A WETDRY mask of a frame (0/1 doubles, Fortran order, as HYDRODATA holds
// it) into physical slot `phys` of its [j][i][slot4] ring.
int upload_mask(rp_ctx* ctx, const double* src, uint8_t* dst, int64_t cnt, int phys) {
    std::vector<uint8_t> m8((size_t)cnt);
    for (int64_t i = 0; i < cnt; i++) {
        if (src[i] != 0.0 && src[i] != 1.0) return fail(ctx, RP_ERR_ARG, "rp_upload_frame: wetdry masks must be 0 or 1");
        m8[(size_t)i] = src[i] != 0.0 ? 1 : 0;
    }
    int rc;
    if ((rc = h2d(ctx, ctx->wd_stage, m8.data(), (size_t)cnt, ctx->s_copy)) != RP_OK) return rc;
    CK(rp::launch_mask_slot(ctx->wd_stage, dst, cnt, phys, ctx->s_copy));
    ctx->launches++;
    return RP_OK;
}

template <typename S>
int upload_frame(rp_ctx* ctx, int32_t ng, int32_t slot, const S* zeta, const S* u, const S* v, const S* w,
                 const S* aks, const S* su, const S* sv, const S* salt = nullptr, const S* temp = nullptr,
                 const S* bustr = nullptr, const S* bvstr = nullptr, const double* wd_rho = nullptr,
                 const double* wd_u = nullptr, const double* wd_v = nullptr, const S* turbaccel = nullptr,
                 const S* turbvort = nullptr, const S* waveaccelu = nullptr, const S* waveaccelv = nullptr) {
    if (!ctx) return RP_ERR_ARG;
    if (ng < 1 || ng > ctx->ngrid) return fail(ctx, RP_ERR_ARG, "rp_upload_frame: grid id out of range");
    if (slot < 1 || slot > 3) return fail(ctx, RP_ERR_ARG, "rp_upload_frame: slot must be 1..3");
    if (!zeta || !u || !v || !w || !aks) return fail(ctx, RP_ERR_ARG, "rp_upload_frame: null field");
    if ((ctx->diag & RP_DIAG_SALTTEMP) && (!salt || !temp))
        return fail(ctx, RP_ERR_ARG, "rp_upload_frame: SaltTempOn needs salt and temp (rp_upload_frame_ext)");
    if ((ctx->diag & RP_DIAG_BOTTOM) && (!bustr || !bvstr))
        return fail(ctx, RP_ERR_ARG, "rp_upload_frame: WriteBottom needs bustr and bvstr (rp_upload_frame_ext)");
    if (ctx->beh.va && (!turbaccel || !turbvort))
        return fail(ctx, RP_ERR_ARG, "rp_upload_frame: Process_VA needs turbaccel and turbvort (rp_upload_frame_desc)");
    if (ctx->beh.wa && (!waveaccelu || !waveaccelv))
        return fail(ctx, RP_ERR_ARG, "rp_upload_frame: Process_WA needs waveaccelu and waveaccelv (rp_upload_frame_desc)");
    if (ctx->wetdry && (!wd_rho || !wd_u || !wd_v))
        return fail(ctx, RP_ERR_ARG, "rp_upload_frame: WETDRY needs the frame's wetdry masks (rp_upload_frame_desc)");
    const bool stokes = ctx->prm.stokes != 0;
    if (stokes && (!su || !sv)) return fail(ctx, RP_ERR_ARG, "rp_upload_frame: stokes on but su/sv null");
    GridBuf& G = ctx->g[ng - 1];
    CK(cudaSetDevice(ctx->device));
    // a physical slot not mapped to any logical slot
    int phys = -1;
    for (int p = 0; p < RP_SLOTS && phys < 0; p++) {
        bool used = false;
        for (int l = 0; l < 3; l++) used = used || (G.map[l] == p);
        if (!used) phys = p;
    }
    if (G.free_recorded[phys]) CK(cudaStreamWaitEvent(ctx->s_copy, G.slot_free[phys], 0));
    const int nx = G.nx, ny = G.ny, N = G.N;
    int rc;
    const bool mx = ctx->mixed;
    if ((rc = upload_field<S>(ctx, zeta, nullptr, G.zeta, nx, ny, 1, phys, mx)) != RP_OK) return rc;
    if ((rc = upload_field<S>(ctx, u, stokes ? su : nullptr, G.u, nx - 1, ny, N, phys, mx, G.qs_u)) != RP_OK)
        return rc;
    if ((rc = upload_field<S>(ctx, v, stokes ? sv : nullptr, G.v, nx, ny - 1, N, phys, mx, G.qs_v)) != RP_OK)
        return rc;
    if ((rc = upload_field<S>(ctx, w, nullptr, G.w, nx, ny, N + 1, phys, mx, G.qs_w)) != RP_OK) return rc;
    if ((rc = upload_field<S>(ctx, aks, nullptr, G.aks, nx, ny, N + 1, phys, mx, G.qs_aks)) != RP_OK) return rc;
    if (ctx->diag & RP_DIAG_SALTTEMP) {
        if ((rc = upload_field<S>(ctx, salt, nullptr, G.salt, nx, ny, N, phys, mx)) != RP_OK) return rc;
        if ((rc = upload_field<S>(ctx, temp, nullptr, G.temp, nx, ny, N, phys, mx)) != RP_OK) return rc;
    }
    if (ctx->diag & RP_DIAG_BOTTOM) {
        if ((rc = upload_field<S>(ctx, bustr, nullptr, G.bustr, nx - 1, ny, 1, phys, mx)) != RP_OK) return rc;
        if ((rc = upload_field<S>(ctx, bvstr, nullptr, G.bvstr, nx, ny - 1, 1, phys, mx)) != RP_OK) return rc;
    }
    if (ctx->beh.va) {
        if ((rc = upload_field<S>(ctx, turbaccel, nullptr, G.turbaccel, nx, ny, N + 1, phys, mx)) != RP_OK) return rc;
        if ((rc = upload_field<S>(ctx, turbvort, nullptr, G.turbvort, nx, ny, N + 1, phys, mx)) != RP_OK) return rc;
    }
    if (ctx->beh.wa) {
        if ((rc = upload_field<S>(ctx, waveaccelu, nullptr, G.waveaccelu, nx, ny, N + 1, phys, mx)) != RP_OK) return rc;
        if ((rc = upload_field<S>(ctx, waveaccelv, nullptr, G.waveaccelv, nx, ny, N + 1, phys, mx)) != RP_OK) return rc;
    }
    if (ctx->wetdry) {
        if ((rc = upload_mask(ctx, wd_rho, G.wd_rho, (int64_t)nx * ny, phys)) != RP_OK) return rc;
        if ((rc = upload_mask(ctx, wd_u, G.wd_u, (int64_t)(nx - 1) * ny, phys)) != RP_OK) return rc;
        if ((rc = upload_mask(ctx, wd_v, G.wd_v, (int64_t)nx * (ny - 1), phys)) != RP_OK) return rc;
    }
    CK(cudaEventRecord(G.slot_ready[phys], ctx->s_copy));
    if (ctx->direct_pending) {                 // the caller's arrays are free again once copied
        CK(cudaEventSynchronize(G.slot_ready[phys]));
        ctx->direct_pending = false;
    }
    G.slot_loaded[phys] = true;
    const int old = G.map[slot - 1];
    G.map[slot - 1] = phys;
    if (old >= 0) {
        // readers of the old physical slot are all queued on the compute stream
        if (mx) {
            // the mixed form reads all four slots of a (point, level) and
            // weighs the spare one 0: clear it (values and scales), after
            // its last reader and before the next upload into it
            const int64_t n2 = (int64_t)nx * ny, nu = (int64_t)(nx - 1) * ny, nv = (int64_t)nx * (ny - 1);
            const struct { void* p; int e; int64_t n; } rings[] = {
                {G.zeta, 4, n2}, {G.u, 2, nu * N}, {G.v, 2, nv * N}, {G.w, 2, n2 * (N + 1)}, {G.aks, 2, n2 * (N + 1)},
                {G.qs_u, 4, N + 1}, {G.qs_v, 4, N + 1}, {G.qs_w, 4, N + 1}, {G.qs_aks, 4, N + 1},
                {G.salt, 4, n2 * N}, {G.temp, 4, n2 * N}, {G.bustr, 4, nu}, {G.bvstr, 4, nv},
                {G.turbaccel, 4, n2 * (N + 1)}, {G.turbvort, 4, n2 * (N + 1)},
                {G.waveaccelu, 4, n2 * (N + 1)}, {G.waveaccelv, 4, n2 * (N + 1)}};
            for (const auto& r : rings) CK(rp::launch_clear_slot(r.p, r.e, r.n, old, ctx->num_sms, ctx->s_comp));
        }
        CK(cudaEventRecord(G.slot_free[old], ctx->s_comp));
        G.free_recorded[old] = true;
        G.slot_loaded[old] = false;
    }
    return RP_OK;
}

// Buffers of the re-sort (once per context).
int sort_buffers(rp_ctx* ctx) {
    if (ctx->sb.keys) return RP_OK;
    RpStepArgs A{};
    A.ngrid = ctx->ngrid;
    fill_grids(ctx, A, 1, 1, 1);
    uint32_t gb[RP_MAXNGRID] = {};
    ctx->sb.nkeys = rp::sort_key_count(A, gb);
    if (ctx->sb.nkeys > rp::kSortMaxKeys)
        return fail(ctx, RP_ERR_UNSUPPORTED, "re-sort: grids exceed 1,048,576 cells in all");
    const size_t cap = (size_t)ctx->cap;
    if (dalloc(&ctx->sb.keys, cap * 4) || dalloc(&ctx->sb.perm, cap * 4) ||
        dalloc(&ctx->sb.hist, (size_t)ctx->sb.nkeys * 4) || dalloc(&ctx->sb.sums, 1024 * 4) ||
        dalloc(&ctx->sb.gbase, sizeof(gb)))
        return fail(ctx, RP_ERR_NOMEM, "re-sort buffers");
    CK(cudaMemcpy(ctx->sb.gbase, gb, sizeof(gb), cudaMemcpyHostToDevice));
    return RP_OK;
}

// An adjoint state block: x, y, z, age, status (doubles), gid (int32),
// isin (int8) for n particles, laid out in one allocation of
// adj_block_bytes(n).
size_t adj_block_bytes(int64_t n) { return (size_t)n * (5 * 8 + 4 + 1) + 64; }

rp::AdjStateDev adj_view(void* base, int64_t n) {
    rp::AdjStateDev s;
    char* p = (char*)base;
    s.x = (double*)p;
    s.y = s.x + n;
    s.z = s.y + n;
    s.age = s.z + n;
    s.status = s.age + n;
    s.gid = (int32_t*)(s.status + n);
    s.isin = (int8_t*)(s.gid + n);
    return s;
}

rp::AdjStateDev adj_ctx_state(rp_ctx* c) {
    rp::AdjStateDev s;
    s.x = c->x; s.y = c->y; s.z = c->z; s.age = c->age; s.status = c->status; s.gid = c->gid; s.isin = c->isin;
    return s;
}

// copy state a -> b (n particles) on stream st
cudaError_t adj_copy(const rp::AdjStateDev& a, const rp::AdjStateDev& b, int64_t n, cudaStream_t st) {
    const size_t d = (size_t)n * 8;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(b.x, a.x, d, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.y, a.y, d, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.z, a.z, d, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.age, a.age, d, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.status, a.status, d, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.gid, a.gid, (size_t)n * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    return cudaMemcpyAsync(b.isin, a.isin, (size_t)n, cudaMemcpyDeviceToDevice, st);
}

// the arguments of step s of the recorded table
void adj_args(rp_ctx* ctx, const rp_adj_step& st, RpStepArgs& A, AdjFrames& F, int64_t n) {
    A = RpStepArgs{};
    fill_params(ctx, A);
    fill_grids(ctx, A, 1, 1, 1);
    A.p.n = n;
    for (int q = 0; q < 3; q++) { A.ex[q] = st.ex[q]; A.ix[q] = st.ix[q]; }
    A.pi = polint_consts(st.ex, st.ix[1]);
    A.ets = st.ets;
    A.step_index = st.step_index;
    A.hook = nullptr;
    const int fr[3] = {st.frame_b, st.frame_c, st.frame_f};
    for (int g = 0; g < ctx->ngrid; g++)
        for (int f = 0; f < 5; f++)
            for (int t = 0; t < 3; t++)
                F.f[g][f][t] = ctx->adj.fst[g][f] + (size_t)(fr[t] - 1) * ctx->adj.fsize[g][f];
}

int adj_upload_field(rp_ctx* ctx, const double* src, const double* add, double* dst, int ni, int nj, int nk) {
    const int64_t total = (int64_t)ni * nj * nk;
    for (int64_t e0 = 0; e0 < total; e0 += kChunkElems) {
        const int64_t cnt = std::min<int64_t>(kChunkElems, total - e0);
        const size_t nb = (size_t)cnt * 8;
        const int h = ctx->pin_next;
        ctx->pin_next ^= 1;
        if (ctx->pin_used[h]) CK(cudaEventSynchronize(ctx->pin_done[h]));
        char* pin = (char*)ctx->pin[h];
        char* ds = (char*)ctx->dstage[h];
        std::memcpy(pin, src + e0, nb);
        if (add) std::memcpy(pin + (size_t)kChunkElems * 8, add + e0, nb);
        CK(cudaMemcpyAsync(ds, pin, add ? (size_t)kChunkElems * 8 + nb : nb, cudaMemcpyHostToDevice, ctx->s_copy));
        CK(rp::launch_adj_store((const double*)ds, add ? (const double*)(ds + (size_t)kChunkElems * 8) : nullptr,
                                dst, ni, nj, nk, e0, cnt, ctx->s_copy));
        ctx->launches++;
        CK(cudaEventRecord(ctx->pin_done[h], ctx->s_copy));
        ctx->pin_used[h] = true;
    }
    return RP_OK;
}

// ini_ROMSPath's particle set-up (ROMSPath.f90:319-432) on the device:
// the particles' fractional indices in every grid, either given (ipos,
// jpos; (n, Ngrid) Fortran order) or by LL2ij from lon/lat, then the
// ownership loop with bounds/zbounds and the initial diagnostics.
int locate(rp_ctx* ctx, int64_t n, const double* ipos, const double* jpos, const double* lon, const double* lat,
           const double* z, const double* dob, int32_t t_b, double* ipos_out, double* jpos_out) {
    if (n < 0 || n > ctx->cap) return fail(ctx, RP_ERR_ARG, "rp_locate_particles: n exceeds numpar");
    if (!z || !dob) return fail(ctx, RP_ERR_ARG, "rp_locate_particles: null array");
    if (t_b < 1 || t_b > 3) return fail(ctx, RP_ERR_ARG, "rp_locate_particles: slot must be 1..3");
    // SaltTempOn reads the initial salinity and temperature from t_c, the
    // slot after t_b (ROMSPath.f90:209-211, 408-427)
    const int32_t t_c = (ctx->diag & RP_DIAG_SALTTEMP) ? t_b % 3 + 1 : t_b;
    for (int k = 0; k < ctx->ngrid; k++)
        if (ctx->g[k].map[t_b - 1] < 0 || ctx->g[k].map[t_c - 1] < 0)
            return fail(ctx, RP_ERR_STATE, "rp_locate_particles: frame slot not loaded");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    const size_t nb = (size_t)n * 8, nbg = nb * ctx->ngrid;
    double *dip = nullptr, *djp = nullptr, *dz = nullptr, *ddob = nullptr, *dlon = nullptr, *dlat = nullptr;
    CK(cudaMalloc(&dip, std::max<size_t>(nbg, 8)));
    CK(cudaMalloc(&djp, std::max<size_t>(nbg, 8)));
    CK(cudaMalloc(&dz, std::max<size_t>(nb, 8)));
    CK(cudaMalloc(&ddob, std::max<size_t>(nb, 8)));
    if (lon) {
        CK(cudaMalloc(&dlon, std::max<size_t>(nb, 8)));
        CK(cudaMalloc(&dlat, std::max<size_t>(nb, 8)));
    }
    int rc = RP_OK;
    cudaError_t e = cudaSuccess;
    if (lon) {
        if (!(rc = h2d(ctx, dlon, lon, nb, s)) && !(rc = h2d(ctx, dlat, lat, nb, s))) {
            // LL2ij reads GRIDS(1)%spherical for every grid (interpolation_module.f90:171)
            const int sph = ctx->g[0].spherical;
            for (int k = 0; k < ctx->ngrid && e == cudaSuccess; k++) {
                const GridBuf& G = ctx->g[k];
                if (sph != 0 && !G.angle) {
                    rc = fail(ctx, RP_ERR_STATE, "rp_locate_lonlat: spherical grids need their angle");
                    break;
                }
                e = rp::launch_ll2ij(G.lon, G.lat, G.angle, G.nx, G.ny, sph, dlon, dlat, n, dip + (size_t)k * n,
                                     djp + (size_t)k * n, ctx->num_sms, s);
                ctx->launches++;
            }
            if (e == cudaSuccess && rc == RP_OK && ipos_out) rc = d2h(ctx, ipos_out, dip, nbg, s);
            if (e == cudaSuccess && rc == RP_OK && jpos_out) rc = d2h(ctx, jpos_out, djp, nbg, s);
        }
    } else {
        if (!(rc = h2d(ctx, dip, ipos, nbg, s))) rc = h2d(ctx, djp, jpos, nbg, s);
    }
    if (rc == RP_OK && e == cudaSuccess && !(rc = h2d(ctx, dz, z, nb, s)) && !(rc = h2d(ctx, ddob, dob, nb, s))) {
        ctx->n = n;
        ctx->permuted = false;
        ctx->since_sort = ctx->resort;
        ctx->state_base = ctx->pid_base;
        RpStepArgs A{};
        fill_params(ctx, A);
        fill_grids(ctx, A, t_b, t_c, t_b);
        for (int k = 0; k < ctx->ngrid; k++) {
            cudaStreamWaitEvent(s, ctx->g[k].slot_ready[ctx->g[k].map[t_b - 1]], 0);
            cudaStreamWaitEvent(s, ctx->g[k].slot_ready[ctx->g[k].map[t_c - 1]], 0);
        }
        e = rp::launch_locate(A, ctx->mixed ? RP_FIELD_F32 : ctx->prm.field_dtype, dip, djp, dz, ddob, s);
        ctx->launches++;
        if (e == cudaSuccess && ctx->mixed) {
            e = rp::launch_mixed_convert(A.p, 0, s);
            ctx->launches++;
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess && rc == RP_OK) rc = fail(ctx, RP_ERR_CUDA, std::string("locate: ") + cudaGetErrorString(e));
    cudaFree(dip); cudaFree(djp); cudaFree(dz); cudaFree(ddob);
    if (dlon) cudaFree(dlon);
    if (dlat) cudaFree(dlat);
    return rc;
}

constexpr int kOutCols = 11;

// Checks, then packs one output record into the device record buffer on
// the compute stream (after the read-back of an earlier asynchronous
// record, which shares the buffer); dev[c] receives each column's address.
int output_pack(rp_ctx* ctx, int64_t n, int32_t mI, double* const host[kOutCols], double* dev[kOutCols]) {
    const bool lon = host[0] || host[1];
    if (n < 0 || n > ctx->n) return fail(ctx, RP_ERR_ARG, "rp_output_record: n exceeds particle count");
    if (lon)
        for (int k = 0; k < ctx->ngrid; k++)
            if (!ctx->g[k].lon) return fail(ctx, RP_ERR_STATE, "rp_output_record: lon/lat need rp_set_grid_lonlat");
    if (((host[6] || host[7]) && !(ctx->diag & RP_DIAG_SALTTEMP)) ||
        ((host[8] || host[9] || host[10]) && !(ctx->diag & RP_DIAG_BOTTOM)))
        return fail(ctx, RP_ERR_STATE, "rp_output_record: that diagnostic is off in this context");
    if ((ctx->diag & RP_DIAG_SALTTEMP_MEAN) && mI < 1)
        return fail(ctx, RP_ERR_ARG, "rp_output_record: SaltTempMean needs the step count mI >= 1");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    if (!ctx->outbuf && dalloc(&ctx->outbuf, (size_t)kOutCols * ctx->cap * 8))
        return fail(ctx, RP_ERR_NOMEM, "rp_output_record: record buffer");
    if (ctx->out_pending) CK(cudaStreamWaitEvent(s, ctx->ev_out_done, 0));
    for (int c = 0; c < kOutCols; c++) dev[c] = host[c] ? ctx->outbuf + (size_t)c * ctx->cap : nullptr;
    rp::OutCols o{dev[0], dev[1], dev[2], dev[3], dev[4], dev[5], dev[6], dev[7], dev[8], dev[9], dev[10]};
    RpStepArgs A{};
    fill_params(ctx, A);
    fill_grids(ctx, A, 1, 1, 1);
    if (ctx->mixed) {                          // the FP64 columns from the compensated FP32 positions
        CK(rp::launch_mixed_convert(A.p, 1, s));
        ctx->launches++;
    }
    CK(rp::launch_output(A, o, ctx->permuted ? 1 : 0, ctx->state_base, n, mI, s));
    ctx->launches++;
    return RP_OK;
}

}  // namespace

extern "C" {

const char* rp_version(void) { return "romspath_b200 0.1 (sm_100a)"; }

int rp_create(const rp_params* params, int32_t ngrid, const rp_grid* grids, rp_ctx** out) {
    if (!params || !grids || !out) return RP_ERR_ARG;
    *out = nullptr;
    const rp_params& p = *params;
    if (ngrid < 1 || ngrid > RP_MAXNGRID || p.numpar < 0 || p.idt <= 0 || p.dt <= 0) return RP_ERR_ARG;
    if (p.behavior != 0 && p.behavior != 1 && p.behavior != 10 && p.behavior != 11) return RP_ERR_UNSUPPORTED;
    if (p.nsb < 0 || p.nsb > 2) return RP_ERR_ARG;
    if (!(p.deltat >= 1.0) || !(p.sub > 0.0)) return RP_ERR_ARG;
    if (p.field_dtype != RP_FIELD_F64 && p.field_dtype != RP_FIELD_F32 && p.field_dtype != RP_FIELD_MIXED &&
        p.field_dtype != RP_FIELD_MIXED_I16)
        return RP_ERR_ARG;
    if (p.reserved[3] & ~(RP_DIAG_SALTTEMP | RP_DIAG_SALTTEMP_MEAN | RP_DIAG_BOTTOM)) return RP_ERR_ARG;
    if (p.reserved[4] != 0 && p.reserved[4] != 1) return RP_ERR_ARG;
    if (p.reserved[0] < 0 || p.reserved[0] > 5) return RP_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p.device || p.device < 0) return RP_ERR_NOEXT;
    rp_ctx* ctx = new rp_ctx();
    ctx->prm = p;
    ctx->ngrid = ngrid;
    ctx->device = p.device;
    ctx->elem = (p.field_dtype == RP_FIELD_F32) ? 4 : 8;
    ctx->mixed = (p.field_dtype == RP_FIELD_MIXED || p.field_dtype == RP_FIELD_MIXED_I16);
    ctx->i16 = (p.field_dtype == RP_FIELD_MIXED_I16);
    ctx->ndraw = 2 + p.idt / (int)p.deltat;
    ctx->wetdry = p.reserved[4] == 1;
    // SaltTempMean applies only with SaltTempOn (ROMSPath.f90:247-257)
    ctx->diag = p.reserved[3] & (RP_DIAG_SALTTEMP | RP_DIAG_BOTTOM);
    if ((p.reserved[3] & RP_DIAG_SALTTEMP_MEAN) && (p.reserved[3] & RP_DIAG_SALTTEMP))
        ctx->diag |= RP_DIAG_SALTTEMP_MEAN;
    auto bail = [&](int code, const std::string& m) {
        std::fprintf(stderr, "rp_create: %s\n", m.c_str());
        free_ctx(ctx);
        return code;
    };
    if (cudaSetDevice(p.device) != cudaSuccess) return bail(RP_ERR_CUDA, "cudaSetDevice failed");
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, p.device);
    for (int k = 0; k < ngrid; k++) {
        const rp_grid& R = grids[k];
        GridBuf& G = ctx->g[k];
        // N >= 2: with one s-level the reference's linint search (interpolation_module.f90:37-47)
        // never ends for a resampling point below the first level
        if (R.xi_rho < 4 || R.eta_rho < 4 || R.n_rho < 2 || R.n_rho > 510)
            return bail(RP_ERR_ARG, "bad grid dims (xi_rho, eta_rho >= 4; 2 <= N <= 510)");
        if (R.vtransform < 1 || R.vtransform > 3) return bail(RP_ERR_ARG, "bad Vtransform");
        if (!R.h || !R.pm || !R.pn || !R.mask_rho || !R.mask_u || !R.mask_v || !R.s_rho || !R.cs_r || !R.s_w || !R.cs_w)
            return bail(RP_ERR_ARG, "null grid array");
        if (ngrid > 1 && (!R.scl || !R.off)) return bail(RP_ERR_ARG, "nested grids need scl/off");
        G.nx = R.xi_rho; G.ny = R.eta_rho; G.N = R.n_rho; G.vtransform = R.vtransform; G.hc = R.hc;
        // the mixed form indexes a grid's fields in 32 bits (corner * levels + level)
        if (ctx->mixed && (int64_t)G.nx * G.ny * std::max(G.N + 1, RP_SLOTS) > (int64_t)INT32_MAX)
            return bail(RP_ERR_UNSUPPORTED, "mixed form: xi_rho * eta_rho * max(N + 1, 4) must be below 2^31");
        const int sw = G.N + 1;
        const int np = (int)((double)sw * p.sub);
        if (np < 4 || np > kMaxNp || np < sw) return bail(RP_ERR_UNSUPPORTED, "spline point count int(s_w*sub) must be in [max(4,s_w), 144]");
        ctx->npmax = std::max(ctx->npmax, np);
        const size_t n2 = (size_t)G.nx * G.ny;
        const size_t nu = (size_t)(G.nx - 1) * G.ny, nv = (size_t)G.nx * (G.ny - 1);
        std::vector<uint8_t> m8(std::max(n2, std::max(nu, nv)));
        auto mask8 = [&](const int32_t* m, size_t cnt) -> bool {
            for (size_t i = 0; i < cnt; i++) {
                if (m[i] != 0 && m[i] != 1) return false;
                m8[i] = (uint8_t)m[i];
            }
            return true;
        };
        if (dalloc(&G.h, n2 * 8) || dalloc(&G.pm, n2 * 8) || dalloc(&G.pn, n2 * 8) ||
            dalloc(&G.sr, G.N * 8) || dalloc(&G.csr, G.N * 8) || dalloc(&G.sw, sw * 8) || dalloc(&G.csw, sw * 8) ||
            dalloc(&G.scs_r, G.N * sizeof(float2)) || dalloc(&G.scs_w, sw * sizeof(float2)) ||
            dalloc(&G.hm, n2 * sizeof(float2)) ||
            dalloc(&G.mrho, n2) || dalloc(&G.mu, nu) || dalloc(&G.mv, nv))
            return bail(RP_ERR_NOMEM, "grid allocation");
        cudaMemcpy(G.h, R.h, n2 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(G.pm, R.pm, n2 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(G.pn, R.pn, n2 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(G.sr, R.s_rho, G.N * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(G.csr, R.cs_r, G.N * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(G.sw, R.s_w, sw * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(G.csw, R.cs_w, sw * 8, cudaMemcpyHostToDevice);
        {
            std::vector<float2> pr(G.N), pw(sw);
            for (int k = 0; k < G.N; k++) pr[k] = make_float2((float)R.s_rho[k], (float)R.cs_r[k]);
            for (int k = 0; k < sw; k++) pw[k] = make_float2((float)R.s_w[k], (float)R.cs_w[k]);
            cudaMemcpy(G.scs_r, pr.data(), G.N * sizeof(float2), cudaMemcpyHostToDevice);
            cudaMemcpy(G.scs_w, pw.data(), sw * sizeof(float2), cudaMemcpyHostToDevice);
        }
        if (!mask8(R.mask_rho, n2)) return bail(RP_ERR_ARG, "mask_rho values must be 0 or 1");
        cudaMemcpy(G.mrho, m8.data(), n2, cudaMemcpyHostToDevice);
        {
            std::vector<float2> hm(n2);
            for (size_t i = 0; i < n2; i++) hm[i] = make_float2((float)R.h[i], (float)m8[i]);
            cudaMemcpy(G.hm, hm.data(), n2 * sizeof(float2), cudaMemcpyHostToDevice);
        }
        if (!mask8(R.mask_u, nu)) return bail(RP_ERR_ARG, "mask_u values must be 0 or 1");
        cudaMemcpy(G.mu, m8.data(), nu, cudaMemcpyHostToDevice);
        if (!mask8(R.mask_v, nv)) return bail(RP_ERR_ARG, "mask_v values must be 0 or 1");
        if (cudaMemcpy(G.mv, m8.data(), nv, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(RP_ERR_CUDA, "grid upload");
        for (int i = 0; i < ngrid; i++) {
            if (ngrid == 1 && !R.scl) {
                G.scl[i][0] = G.scl[i][1] = 1.0;
                G.off[i][0] = G.off[i][1] = 0.0;
            } else {
                G.scl[i][0] = R.scl[i]; G.scl[i][1] = R.scl[ngrid + i];
                G.off[i][0] = R.off[i]; G.off[i][1] = R.off[ngrid + i];
            }
        }
        // bytes per (point, level) over the ring: zeta and the 3-D fields
        const size_t ez = (size_t)(ctx->mixed ? 4 : ctx->elem) * RP_SLOTS;
        const size_t e = (size_t)(ctx->mixed ? 2 : ctx->elem) * RP_SLOTS;
        if (dalloc(&G.zeta, n2 * ez) || dalloc(&G.u, nu * G.N * e) || dalloc(&G.v, nv * G.N * e) ||
            dalloc(&G.w, n2 * sw * e) || dalloc(&G.aks, n2 * sw * e))
            return bail(RP_ERR_NOMEM, "frame ring allocation");
        cudaMemset(G.zeta, 0, n2 * ez);
        cudaMemset(G.u, 0, nu * G.N * e);
        cudaMemset(G.v, 0, nv * G.N * e);
        cudaMemset(G.w, 0, n2 * sw * e);
        cudaMemset(G.aks, 0, n2 * sw * e);
        // the diagnostics' fields: FP32 in the mixed form
        const size_t ed = (size_t)(ctx->mixed ? 4 : ctx->elem) * RP_SLOTS;
        if (ctx->diag & RP_DIAG_SALTTEMP) {
            if (dalloc(&G.salt, n2 * G.N * ed) || dalloc(&G.temp, n2 * G.N * ed))
                return bail(RP_ERR_NOMEM, "salt/temp ring allocation");
            cudaMemset(G.salt, 0, n2 * G.N * ed);
            cudaMemset(G.temp, 0, n2 * G.N * ed);
        }
        if (ctx->wetdry) {
            if (dalloc(&G.wd_rho, n2 * RP_SLOTS) || dalloc(&G.wd_u, nu * RP_SLOTS) || dalloc(&G.wd_v, nv * RP_SLOTS))
                return bail(RP_ERR_NOMEM, "wetdry mask ring allocation");
            cudaMemset(G.wd_rho, 0, n2 * RP_SLOTS);
            cudaMemset(G.wd_u, 0, nu * RP_SLOTS);
            cudaMemset(G.wd_v, 0, nv * RP_SLOTS);
        }
        if (ctx->diag & RP_DIAG_BOTTOM) {
            if (dalloc(&G.bustr, nu * ed) || dalloc(&G.bvstr, nv * ed))
                return bail(RP_ERR_NOMEM, "bottom stress ring allocation");
            cudaMemset(G.bustr, 0, nu * ed);
            cudaMemset(G.bvstr, 0, nv * ed);
        }
        if (ctx->mixed) {
            const size_t qn = (size_t)RP_SLOTS * sw * 4;
            if (dalloc(&G.qs_u, qn) || dalloc(&G.qs_v, qn) || dalloc(&G.qs_w, qn) || dalloc(&G.qs_aks, qn))
                return bail(RP_ERR_NOMEM, "scale allocation");
            cudaMemset(G.qs_u, 0, qn);
            cudaMemset(G.qs_v, 0, qn);
            cudaMemset(G.qs_w, 0, qn);
            cudaMemset(G.qs_aks, 0, qn);
        }
        for (int s = 0; s < RP_SLOTS; s++) {
            if (cudaEventCreateWithFlags(&G.slot_free[s], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&G.slot_ready[s], cudaEventDisableTiming) != cudaSuccess)
                return bail(RP_ERR_CUDA, "event creation");
        }
    }
    const size_t cap = (size_t)std::max(p.numpar, 1);
    ctx->cap = (int64_t)cap;
    if (ctx->mixed) {
        size_t fmax = 0, lmax = 0;
        for (int k = 0; k < ngrid; k++) {
            fmax = std::max(fmax, (size_t)ctx->g[k].nx * ctx->g[k].ny * (ctx->g[k].N + 1));
            lmax = std::max(lmax, (size_t)ctx->g[k].N + 1);
        }
        if (dalloc(&ctx->x32, cap * 4) || dalloc(&ctx->y32, cap * 4) || dalloc(&ctx->z32, cap * 4) ||
            dalloc(&ctx->cx, cap * 4) || dalloc(&ctx->cy, cap * 4) || dalloc(&ctx->cz, cap * 4) ||
            dalloc(&ctx->qwarm, cap * 8) || dalloc(&ctx->gwarm, cap * 8) || dalloc(&ctx->qwarm2, cap * 4) ||
            dalloc(&ctx->ftmp, fmax * 4) || dalloc(&ctx->qmax, lmax * 4))
            return bail(RP_ERR_NOMEM, "mixed-form allocation");
    }
    if (dalloc(&ctx->x, cap * 8) || dalloc(&ctx->y, cap * 8) || dalloc(&ctx->z, cap * 8) ||
        dalloc(&ctx->age, cap * 8) || dalloc(&ctx->dob, cap * 8) || dalloc(&ctx->status, cap * 8) ||
        dalloc(&ctx->wd, cap * 8) || dalloc(&ctx->zeta, cap * 8) || dalloc(&ctx->bath, cap * 8) ||
        dalloc(&ctx->gid, cap * 4) || dalloc(&ctx->isin, cap) || dalloc(&ctx->pid, cap * 4) ||
        dalloc(&ctx->flags, cap * 4) || dalloc(&ctx->tmp_gid, cap * 8) || dalloc(&ctx->tmp_isin, cap * 4) ||
        dalloc(&ctx->turbv, cap * 12))
        return bail(RP_ERR_NOMEM, "particle state allocation");
    if (ctx->wetdry) {
        size_t mmax = 0;
        for (int k = 0; k < ngrid; k++) mmax = std::max(mmax, (size_t)ctx->g[k].nx * ctx->g[k].ny);
        if (dalloc(&ctx->wd_stage, mmax)) return bail(RP_ERR_NOMEM, "wetdry staging");
    }
    if ((ctx->diag & RP_DIAG_SALTTEMP) && (dalloc(&ctx->d_salt, cap * 8) || dalloc(&ctx->d_temp, cap * 8)))
        return bail(RP_ERR_NOMEM, "diagnostics allocation");
    if ((ctx->diag & RP_DIAG_SALTTEMP_MEAN) && (dalloc(&ctx->d_mean_salt, cap * 8) || dalloc(&ctx->d_mean_temp, cap * 8)))
        return bail(RP_ERR_NOMEM, "diagnostics allocation");
    if ((ctx->diag & RP_DIAG_BOTTOM) &&
        (dalloc(&ctx->d_hob, cap * 8) || dalloc(&ctx->d_bustr, cap * 8) || dalloc(&ctx->d_bvstr, cap * 8)))
        return bail(RP_ERR_NOMEM, "diagnostics allocation");
    ctx->resort = p.reserved[1] > 0 ? p.reserved[1] : 0;
    if (ctx->resort) {
        const int rc = sort_buffers(ctx);
        if (rc != RP_OK) return bail(rc, ctx->err);
    }
    const size_t half = (size_t)kChunkElems * 8 * 2;
    for (int h = 0; h < 2; h++) {
        if (cudaHostAlloc(&ctx->pin[h], half, cudaHostAllocDefault) != cudaSuccess)
            return bail(RP_ERR_NOMEM, "pinned staging");
        if (dalloc(&ctx->dstage[h], half)) return bail(RP_ERR_NOMEM, "device staging");
        if (cudaEventCreateWithFlags(&ctx->pin_done[h], cudaEventDisableTiming) != cudaSuccess)
            return bail(RP_ERR_CUDA, "event creation");
    }
    if (cudaStreamCreateWithFlags(&ctx->s_comp, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->s_copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_packed, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_out_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_na_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_na_out, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess)
        return bail(RP_ERR_CUDA, "stream/event creation");
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(RP_ERR_CUDA, "initial upload");
    *out = ctx;
    return RP_OK;
}

int rp_destroy(rp_ctx* ctx) {
    if (!ctx) return RP_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->s_comp) cudaStreamSynchronize(ctx->s_comp);
    if (ctx->s_copy) cudaStreamSynchronize(ctx->s_copy);
    free_ctx(ctx);
    return RP_OK;
}

int rp_last_error(rp_ctx* ctx, char* buf, int32_t len) {
    if (!ctx || !buf || len <= 0) return RP_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", ctx->err.c_str());
    return RP_OK;
}

int rp_upload_frame(rp_ctx* ctx, int32_t ng, int32_t slot, const double* zeta, const double* u, const double* v,
                    const double* w, const double* aks, const double* su, const double* sv) {
    return upload_frame<double>(ctx, ng, slot, zeta, u, v, w, aks, su, sv);
}

int rp_upload_frame_f32(rp_ctx* ctx, int32_t ng, int32_t slot, const float* zeta, const float* u, const float* v,
                        const float* w, const float* aks, const float* su, const float* sv) {
    return upload_frame<float>(ctx, ng, slot, zeta, u, v, w, aks, su, sv);
}

int rp_upload_frame_desc(rp_ctx* ctx, int32_t ng, int32_t slot, const rp_frame* f) {
    if (!ctx || !f) return RP_ERR_ARG;
    if (f->f32)
        return upload_frame<float>(ctx, ng, slot, (const float*)f->zeta, (const float*)f->u, (const float*)f->v,
                                   (const float*)f->w, (const float*)f->aks, (const float*)f->su, (const float*)f->sv,
                                   (const float*)f->salt, (const float*)f->temp, (const float*)f->bustr,
                                   (const float*)f->bvstr, f->wetdry_rho, f->wetdry_u, f->wetdry_v,
                                   (const float*)f->turbaccel, (const float*)f->turbvort, (const float*)f->waveaccelu,
                                   (const float*)f->waveaccelv);
    return upload_frame<double>(ctx, ng, slot, (const double*)f->zeta, (const double*)f->u, (const double*)f->v,
                                (const double*)f->w, (const double*)f->aks, (const double*)f->su, (const double*)f->sv,
                                (const double*)f->salt, (const double*)f->temp, (const double*)f->bustr,
                                (const double*)f->bvstr, f->wetdry_rho, f->wetdry_u, f->wetdry_v,
                                (const double*)f->turbaccel, (const double*)f->turbvort, (const double*)f->waveaccelu,
                                (const double*)f->waveaccelv);
}

int rp_upload_frame_ext(rp_ctx* ctx, int32_t ng, int32_t slot, const double* zeta, const double* u, const double* v,
                        const double* w, const double* aks, const double* su, const double* sv, const double* salt,
                        const double* temp, const double* bustr, const double* bvstr) {
    return upload_frame<double>(ctx, ng, slot, zeta, u, v, w, aks, su, sv, salt, temp, bustr, bvstr);
}

int rp_upload_frame_ext_f32(rp_ctx* ctx, int32_t ng, int32_t slot, const float* zeta, const float* u,
                            const float* v, const float* w, const float* aks, const float* su, const float* sv,
                            const float* salt, const float* temp, const float* bustr, const float* bvstr) {
    return upload_frame<float>(ctx, ng, slot, zeta, u, v, w, aks, su, sv, salt, temp, bustr, bvstr);
}

int rp_set_particles(rp_ctx* ctx, int64_t n, const double* x, const double* y, const double* z,
                     const double* dob, const double* age, const double* status, const double* gid,
                     const int32_t* isin) {
    if (!ctx) return RP_ERR_ARG;
    if (n < 0 || n > ctx->cap) return fail(ctx, RP_ERR_ARG, "rp_set_particles: n exceeds numpar");
    if (!x || !y || !z || !dob || !age || !status || !gid || !isin)
        return fail(ctx, RP_ERR_ARG, "rp_set_particles: null column");
    for (int64_t i = 0; i < n; i++) {
        const int gi = (int)gid[i];
        if (gi < 1 || gi > ctx->ngrid) return fail(ctx, RP_ERR_ARG, "rp_set_particles: grid id out of range");
    }
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    int rc;
    const size_t b8 = (size_t)n * 8;
    if ((rc = h2d(ctx, ctx->x, x, b8, s)) || (rc = h2d(ctx, ctx->y, y, b8, s)) || (rc = h2d(ctx, ctx->z, z, b8, s)) ||
        (rc = h2d(ctx, ctx->dob, dob, b8, s)) || (rc = h2d(ctx, ctx->age, age, b8, s)) ||
        (rc = h2d(ctx, ctx->status, status, b8, s)) || (rc = h2d(ctx, ctx->tmp_gid, gid, b8, s)) ||
        (rc = h2d(ctx, ctx->tmp_isin, isin, (size_t)n * 4, s)))
        return rc;
    ctx->n = n;
    ctx->permuted = false;
    ctx->since_sort = ctx->resort;
    ctx->state_base = ctx->pid_base;
    RpParticlesDev P = particles_dev(ctx);
    CK(rp::launch_state_from_host(P, ctx->tmp_gid, ctx->tmp_isin, ctx->pid_base, s));
    ctx->launches++;
    if (ctx->mixed) {
        CK(rp::launch_mixed_convert(P, 0, s));
        ctx->launches++;
    }
    CK(cudaMemsetAsync(ctx->wd, 0, b8, s));
    CK(cudaMemsetAsync(ctx->zeta, 0, b8, s));
    CK(cudaMemsetAsync(ctx->bath, 0, b8, s));
    CK(cudaStreamSynchronize(s));
    return RP_OK;
}

int rp_locate_particles(rp_ctx* ctx, int64_t n, const double* ipos, const double* jpos, const double* z,
                        const double* dob, int32_t t_b) {
    if (!ctx) return RP_ERR_ARG;
    if (!ipos || !jpos) return fail(ctx, RP_ERR_ARG, "rp_locate_particles: null array");
    return locate(ctx, n, ipos, jpos, nullptr, nullptr, z, dob, t_b, nullptr, nullptr);
}

int rp_locate_lonlat(rp_ctx* ctx, int64_t n, const double* lon, const double* lat, const double* z, const double* dob,
                     int32_t t_b, double* ipos_out, double* jpos_out) {
    if (!ctx) return RP_ERR_ARG;
    if (!lon || !lat) return fail(ctx, RP_ERR_ARG, "rp_locate_lonlat: null array");
    for (int k = 0; k < ctx->ngrid; k++) {
        if (!ctx->g[k].lon) return fail(ctx, RP_ERR_STATE, "rp_locate_lonlat: lon/lat need rp_set_grid_lonlat");
        if (ctx->g[k].spherical < 0) return fail(ctx, RP_ERR_STATE, "rp_locate_lonlat: rp_set_grid_angle first");
    }
    return locate(ctx, n, nullptr, nullptr, lon, lat, z, dob, t_b, ipos_out, jpos_out);
}

}  // extern "C"

namespace {

// Checks of one internal step's arguments (rp_step / rp_step_n).
int step_check(rp_ctx* ctx, const double* ex, const double* ix, int32_t t_b, int32_t t_c, int32_t t_f, int64_t k) {
    if (!ex || !ix) return RP_ERR_ARG;
    if (t_b < 1 || t_b > 3 || t_c < 1 || t_c > 3 || t_f < 1 || t_f > 3)
        return fail(ctx, RP_ERR_ARG, "rp_step: slots must be 1..3");
    for (int g = 0; g < ctx->ngrid; g++) {
        const GridBuf& G = ctx->g[g];
        if (G.map[t_b - 1] < 0 || G.map[t_c - 1] < 0 || G.map[t_f - 1] < 0)
            return fail(ctx, RP_ERR_STATE, "rp_step: a frame slot was never loaded");
    }
    if (ctx->hook && ctx->hook_pos + k >= ctx->hook_steps)
        return fail(ctx, RP_ERR_STATE, "rp_step: noise hook exhausted");
    if (ctx->prm.behavior != 0 && !ctx->beh_set)
        return fail(ctx, RP_ERR_STATE, "rp_step: Behavior needs rp_set_behavior first");
    return RP_OK;
}

// The compute stream waits for the uploads of the slots a step reads.
int step_waits(rp_ctx* ctx, int32_t t_b, int32_t t_c, int32_t t_f) {
    for (int g = 0; g < ctx->ngrid; g++) {
        const GridBuf& G = ctx->g[g];
        const int used[3] = {G.map[t_b - 1], G.map[t_c - 1], G.map[t_f - 1]};
        for (int q = 0; q < 3; q++) CK(cudaStreamWaitEvent(ctx->s_comp, G.slot_ready[used[q]], 0));
    }
    return RP_OK;
}

// The launches of one internal step on the compute stream (re-sort when
// due, then the step kernels); advances the step counter and the hook.
int step_launch(rp_ctx* ctx, const double ex[3], const double ix[3], int32_t ets, int32_t t_b, int32_t t_c,
                int32_t t_f, int* nl) {
    cudaStream_t s = ctx->s_comp;
    RpStepArgs A{};
    fill_params(ctx, A);
    fill_grids(ctx, A, t_b, t_c, t_f);
    for (int q = 0; q < 3; q++) { A.ex[q] = ex[q]; A.ix[q] = ix[q]; }
    A.pi = polint_consts(ex, ix[1]);
    lagrange_weights(ex, ix[1], ets, A.lw);
    slot_weights(A, ctx->ngrid);
    A.ets = ets;
    A.step_index = ctx->step_index;
    A.hook = ctx->hook ? ctx->hook + ctx->hook_pos * ctx->n * ctx->ndraw : nullptr;
    if (ctx->resort && ctx->n > 0 && ctx->since_sort >= ctx->resort) {
        CK(rp::launch_sort(A, ctx->mixed, ctx->sb, ctx->turbv, s, nl));
        ctx->permuted = true;
        ctx->since_sort = 0;
    }
    ctx->since_sort++;
    if (ctx->n > 0 && ctx->mixed)
        CK(rp::launch_step_mixed(A, ctx->npmax, ctx->i16, (float*)ctx->turbv, ctx->prm.reserved[0], s,
                                 ctx->num_sms, nl));
    else if (ctx->n > 0)
        CK(rp::launch_step(A, ctx->prm.field_dtype, ctx->npmax, ctx->turbv, ctx->prm.reserved[0] == 1 ? 0 : 1, s,
                           ctx->num_sms, nl));
    ctx->step_index++;
    if (ctx->hook) ctx->hook_pos++;
    return RP_OK;
}

}  // namespace

extern "C" {

int rp_step(rp_ctx* ctx, const double ex[3], const double ix[3], int32_t ets, int32_t t_b, int32_t t_c,
            int32_t t_f) {
    if (!ctx) return RP_ERR_ARG;
    int rc;
    if ((rc = step_check(ctx, ex, ix, t_b, t_c, t_f, 0)) != RP_OK) return rc;
    CK(cudaSetDevice(ctx->device));
    if ((rc = step_waits(ctx, t_b, t_c, t_f)) != RP_OK) return rc;
    int nl = 0;
    CK(cudaEventRecord(ctx->ev0, ctx->s_comp));
    if ((rc = step_launch(ctx, ex, ix, ets, t_b, t_c, t_f, &nl)) != RP_OK) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->s_comp));
    ctx->timed = true;
    ctx->last_kernels = nl;
    ctx->launches += nl;
    return RP_OK;
}

int rp_step_n(rp_ctx* ctx, int32_t nsteps, const double* ex, const double* ix, const int32_t* ets,
              const int32_t* t_b, const int32_t* t_c, const int32_t* t_f) {
    if (!ctx || !ex || !ix || !ets || !t_b || !t_c || !t_f) return RP_ERR_ARG;
    if (nsteps < 1) return fail(ctx, RP_ERR_ARG, "rp_step_n: nsteps >= 1");
    int rc;
    for (int k = 0; k < nsteps; k++)
        if ((rc = step_check(ctx, ex + 3 * k, ix + 3 * k, t_b[k], t_c[k], t_f[k], k)) != RP_OK) return rc;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    for (int k = 0; k < nsteps; k++)
        if ((rc = step_waits(ctx, t_b[k], t_c[k], t_f[k])) != RP_OK) return rc;
    // capture this call's launches; the graph of the previous call is
    // updated in place when its shape is the same
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int nl = 0;
    for (int k = 0; k < nsteps && rc == RP_OK; k++)
        rc = step_launch(ctx, ex + 3 * k, ix + 3 * k, ets[k], t_b[k], t_c[k], t_f[k], &nl);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (rc != RP_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return fail(ctx, RP_ERR_CUDA, std::string("rp_step_n: capture: ") + cudaGetErrorString(ec));
    bool updated = false;
    if (ctx->gexec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ctx->gexec, graph, &info) == cudaSuccess) {
            updated = true;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(ctx->gexec);
            ctx->gexec = nullptr;
        }
    }
    cudaError_t e = cudaSuccess;
    if (!updated) e = cudaGraphInstantiate(&ctx->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        ctx->gexec = nullptr;
        return fail(ctx, RP_ERR_CUDA, std::string("rp_step_n: instantiate: ") + cudaGetErrorString(e));
    }
    CK(cudaEventRecord(ctx->ev0, s));
    CK(cudaGraphLaunch(ctx->gexec, s));
    CK(cudaEventRecord(ctx->ev1, s));
    ctx->timed = true;
    ctx->last_kernels = nl;
    ctx->launches += nl;
    return RP_OK;
}

int rp_step_noalloc(rp_ctx* ctx, const rp_device_state* st, const double ex[3], const double ix[3], int32_t ets,
                    int32_t t_b, int32_t t_c, int32_t t_f) {
    if (!ctx || !st || !ex || !ix) return RP_ERR_ARG;
    if (st->n < 0 || st->n > rp::kNoallocMaxParticles)
        return fail(ctx, RP_ERR_ARG, "rp_step_noalloc: state->n exceeds RP_NOALLOC_MAX_PARTICLES (1048576)");
    if (ctx->npmax > 128)
        return fail(ctx, RP_ERR_UNSUPPORTED, "rp_step_noalloc: int(s_w*sub) must be <= 128");
    if (ctx->mixed) return fail(ctx, RP_ERR_UNSUPPORTED, "rp_step_noalloc: not available in the mixed form");
    if (ctx->diag) return fail(ctx, RP_ERR_UNSUPPORTED, "rp_step_noalloc: the diagnostics need the context's state");
    if (ctx->prm.behavior != 0 || ctx->beh.va || ctx->beh.wa)
        return fail(ctx, RP_ERR_UNSUPPORTED, "rp_step_noalloc: behave needs the context's state");
    if (!st->x || !st->y || !st->z || !st->age || !st->dob || !st->status || !st->wd || !st->zeta || !st->bath ||
        !st->gid || !st->isin || !st->pid || !st->flags)
        return fail(ctx, RP_ERR_ARG, "rp_step_noalloc: null state column");
    if (t_b < 1 || t_b > 3 || t_c < 1 || t_c > 3 || t_f < 1 || t_f > 3)
        return fail(ctx, RP_ERR_ARG, "rp_step_noalloc: slots must be 1..3");
    if (ctx->hook) return fail(ctx, RP_ERR_STATE, "rp_step_noalloc: the noise hook is not supported");
    for (int k = 0; k < ctx->ngrid; k++) {
        const GridBuf& G = ctx->g[k];
        if (G.map[t_b - 1] < 0 || G.map[t_c - 1] < 0 || G.map[t_f - 1] < 0)
            return fail(ctx, RP_ERR_STATE, "rp_step_noalloc: a frame slot was never loaded");
    }
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    RpStepArgs A{};
    fill_params(ctx, A);
    fill_grids(ctx, A, t_b, t_c, t_f);
    A.p.n = st->n;
    A.p.x = st->x; A.p.y = st->y; A.p.z = st->z; A.p.age = st->age; A.p.dob = st->dob;
    A.p.status = st->status; A.p.wd = st->wd; A.p.zeta = st->zeta; A.p.bath = st->bath;
    A.p.gid = st->gid; A.p.isin = st->isin; A.p.pid = st->pid; A.p.flags = st->flags;
    for (int q = 0; q < 3; q++) { A.ex[q] = ex[q]; A.ix[q] = ix[q]; }
    A.pi = polint_consts(ex, ix[1]);
    lagrange_weights(ex, ix[1], ets, A.lw);
    slot_weights(A, ctx->ngrid);
    A.ets = ets;
    A.step_index = ctx->step_index;
    A.hook = nullptr;
    for (int k = 0; k < ctx->ngrid; k++) {
        const GridBuf& G = ctx->g[k];
        const int used[3] = {G.map[t_b - 1], G.map[t_c - 1], G.map[t_f - 1]};
        for (int q = 0; q < 3; q++) CK(cudaStreamWaitEvent(s, G.slot_ready[used[q]], 0));
    }
    // order the step after the caller's queued work on its stream (NULL:
    // the legacy default stream), and the caller's later work after the step
    cudaStream_t cs = static_cast<cudaStream_t>(st->stream);
    const bool other = cs != s;
    if (other) {
        CK(cudaEventRecord(ctx->ev_na_in, cs));
        CK(cudaStreamWaitEvent(s, ctx->ev_na_in, 0));
    }
    int nl = 0;
    if (st->n > 0)
        CK(rp::launch_step_noalloc(A, ctx->prm.field_dtype, ctx->npmax, ctx->device, s, ctx->num_sms, &nl));
    if (other) {
        CK(cudaEventRecord(ctx->ev_na_out, s));
        CK(cudaStreamWaitEvent(cs, ctx->ev_na_out, 0));
    }
    ctx->launches += nl;
    ctx->step_index++;
    return RP_OK;
}

int rp_get_particles(rp_ctx* ctx, int64_t n, double* x, double* y, double* z, double* age, double* status,
                     double* gid, int32_t* isin, double* wd, double* zeta, double* bath, uint32_t* flags) {
    if (!ctx) return RP_ERR_ARG;
    if (n < 0 || n > ctx->n) return fail(ctx, RP_ERR_ARG, "rp_get_particles: n exceeds particle count");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    // re-sorted columns are converted whole and returned in the caller's
    // order (particle k = id - id base)
    const int64_t nc = ctx->permuted ? ctx->n : n;
    if (ctx->mixed && (x || y || z)) {
        RpParticlesDev P = particles_dev(ctx);
        P.n = nc;
        CK(rp::launch_mixed_convert(P, 1, s));
        ctx->launches++;
    }
    if (gid || isin) {
        RpParticlesDev P = particles_dev(ctx);
        P.n = nc;
        CK(rp::launch_state_to_host(P, ctx->tmp_gid, ctx->tmp_isin, s));
        ctx->launches++;
    }
    auto col = [&](void* dst, const void* src, int elem) -> int {
        if (!dst) return RP_OK;
        const size_t bytes = (size_t)n * elem;
        if (!ctx->permuted) return d2h(ctx, dst, src, bytes, s);
        CK(rp::launch_unsort(elem, src, ctx->turbv, ctx->pid, ctx->state_base, ctx->n, n, s));
        ctx->launches++;
        return d2h(ctx, dst, ctx->turbv, bytes, s);
    };
    int rc;
    if ((rc = col(x, ctx->x, 8)) || (rc = col(y, ctx->y, 8)) || (rc = col(z, ctx->z, 8)) ||
        (rc = col(age, ctx->age, 8)) || (rc = col(status, ctx->status, 8)) || (rc = col(gid, ctx->tmp_gid, 8)) ||
        (rc = col(isin, ctx->tmp_isin, 4)) || (rc = col(wd, ctx->wd, 8)) || (rc = col(zeta, ctx->zeta, 8)) ||
        (rc = col(bath, ctx->bath, 8)) || (rc = col(flags, ctx->flags, 4)))
        return rc;
    return RP_OK;
}

int rp_get_diagnostics(rp_ctx* ctx, int64_t n, double* salt, double* temp, double* mean_salt, double* mean_temp,
                       double* hob, double* bustr, double* bvstr) {
    if (!ctx) return RP_ERR_ARG;
    if (n < 0 || n > ctx->n) return fail(ctx, RP_ERR_ARG, "rp_get_diagnostics: n exceeds particle count");
    if (((salt || temp) && !ctx->d_salt) || ((mean_salt || mean_temp) && !ctx->d_mean_salt) ||
        ((hob || bustr || bvstr) && !ctx->d_hob))
        return fail(ctx, RP_ERR_STATE, "rp_get_diagnostics: that diagnostic is off in this context");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    auto col = [&](double* dst, const double* src) -> int {
        if (!dst) return RP_OK;
        const size_t bytes = (size_t)n * 8;
        if (!ctx->permuted) return d2h(ctx, dst, src, bytes, s);
        CK(rp::launch_unsort(8, src, ctx->turbv, ctx->pid, ctx->state_base, ctx->n, n, s));
        ctx->launches++;
        return d2h(ctx, dst, ctx->turbv, bytes, s);
    };
    int rc;
    if ((rc = col(salt, ctx->d_salt)) || (rc = col(temp, ctx->d_temp)) || (rc = col(mean_salt, ctx->d_mean_salt)) ||
        (rc = col(mean_temp, ctx->d_mean_temp)) || (rc = col(hob, ctx->d_hob)) || (rc = col(bustr, ctx->d_bustr)) ||
        (rc = col(bvstr, ctx->d_bvstr)))
        return rc;
    return RP_OK;
}

int rp_set_grid_lonlat(rp_ctx* ctx, int32_t ng, const double* lon_rho, const double* lat_rho) {
    if (!ctx) return RP_ERR_ARG;
    if (ng < 1 || ng > ctx->ngrid) return fail(ctx, RP_ERR_ARG, "rp_set_grid_lonlat: grid id out of range");
    if (!lon_rho || !lat_rho) return fail(ctx, RP_ERR_ARG, "rp_set_grid_lonlat: null array");
    CK(cudaSetDevice(ctx->device));
    GridBuf& G = ctx->g[ng - 1];
    const size_t bytes = (size_t)G.nx * G.ny * 8;
    if (!G.lon && (dalloc(&G.lon, bytes) || dalloc(&G.lat, bytes)))
        return fail(ctx, RP_ERR_NOMEM, "rp_set_grid_lonlat: allocation");
    // the step kernels never read these; the copy is ordered before the
    // next output record on the compute stream
    int rc;
    if ((rc = h2d(ctx, G.lon, lon_rho, bytes, ctx->s_comp)) || (rc = h2d(ctx, G.lat, lat_rho, bytes, ctx->s_comp)))
        return rc;
    CK(cudaStreamSynchronize(ctx->s_comp));
    return RP_OK;
}

int rp_set_grid_angle(rp_ctx* ctx, int32_t ng, const double* angle, int32_t spherical) {
    if (!ctx) return RP_ERR_ARG;
    if (ng < 1 || ng > ctx->ngrid) return fail(ctx, RP_ERR_ARG, "rp_set_grid_angle: grid id out of range");
    if (spherical != 0 && spherical != 1) return fail(ctx, RP_ERR_ARG, "rp_set_grid_angle: spherical must be 0 or 1");
    GridBuf& G = ctx->g[ng - 1];
    if (angle) {
        CK(cudaSetDevice(ctx->device));
        const size_t bytes = (size_t)G.nx * G.ny * 8;
        if (!G.angle && dalloc(&G.angle, bytes)) return fail(ctx, RP_ERR_NOMEM, "rp_set_grid_angle: allocation");
        int rc;
        if ((rc = h2d(ctx, G.angle, angle, bytes, ctx->s_comp)) != RP_OK) return rc;
        CK(cudaStreamSynchronize(ctx->s_comp));
    }
    G.spherical = spherical;
    return RP_OK;
}

int rp_output_record(rp_ctx* ctx, int64_t n, int32_t mI, double* lon, double* lat, double* zp, double* age,
                     double* status, double* gid, double* salt, double* temp, double* hob, double* bustr,
                     double* bvstr) {
    if (!ctx) return RP_ERR_ARG;
    double* host[kOutCols] = {lon, lat, zp, age, status, gid, salt, temp, hob, bustr, bvstr};
    double* dev[kOutCols];
    int rc;
    if ((rc = output_pack(ctx, n, mI, host, dev)) != RP_OK) return rc;
    for (int c = 0; c < kOutCols; c++) {
        if (!host[c]) continue;
        if ((rc = d2h(ctx, host[c], dev[c], (size_t)n * 8, ctx->s_comp)) != RP_OK) return rc;
    }
    return RP_OK;
}

int rp_output_record_async(rp_ctx* ctx, int64_t n, int32_t mI, double* lon, double* lat, double* zp,
                           double* age, double* status, double* gid, double* salt, double* temp, double* hob,
                           double* bustr, double* bvstr) {
    if (!ctx) return RP_ERR_ARG;
    double* host[kOutCols] = {lon, lat, zp, age, status, gid, salt, temp, hob, bustr, bvstr};
    for (int c = 0; c < kOutCols; c++)
        if (host[c] && n > 0 && !is_pinned(host[c]))
            return fail(ctx, RP_ERR_ARG, "rp_output_record_async: the arrays must be page-locked");
    double* dev[kOutCols];
    int rc;
    if ((rc = output_pack(ctx, n, mI, host, dev)) != RP_OK) return rc;
    // the copies run on their own stream once the record is packed; the
    // steps enqueued next run meanwhile
    CK(cudaEventRecord(ctx->ev_packed, ctx->s_comp));
    CK(cudaStreamWaitEvent(ctx->s_out, ctx->ev_packed, 0));
    for (int c = 0; c < kOutCols; c++) {
        if (!host[c] || n == 0) continue;
        CK(cudaMemcpyAsync(host[c], dev[c], (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->s_out));
    }
    CK(cudaEventRecord(ctx->ev_out_done, ctx->s_out));
    ctx->out_pending = true;
    return RP_OK;
}

int rp_output_wait(rp_ctx* ctx) {
    if (!ctx) return RP_ERR_ARG;
    if (!ctx->out_pending) return RP_OK;
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventSynchronize(ctx->ev_out_done));
    ctx->out_pending = false;
    return RP_OK;
}

int rp_set_behavior(rp_ctx* ctx, const rp_behavior* b) {
    if (!ctx || !b) return RP_ERR_ARG;
    if (b->behavior != ctx->prm.behavior)
        return fail(ctx, RP_ERR_ARG, "rp_set_behavior: behavior differs from rp_params.behavior");
    if (b->va_flag < 0 || b->va_flag > 2) return fail(ctx, RP_ERR_ARG, "rp_set_behavior: va_flag must be 0, 1 or 2");
    if ((b->process_va || b->process_wa) && !(b->initsize > 0.0))
        return fail(ctx, RP_ERR_ARG, "rp_set_behavior: initsize must be > 0");
    for (int k = 0; k < ctx->ngrid; k++)
        for (int q = 0; q < 3; q++)
            if (ctx->g[k].map[q] >= 0)
                return fail(ctx, RP_ERR_STATE, "rp_set_behavior: call before the first frame upload");
    if (ctx->hook) return fail(ctx, RP_ERR_STATE, "rp_set_behavior: call before rp_set_noise_hook");
    CK(cudaSetDevice(ctx->device));
    RpBehaviorDev d{};
    d.behavior = b->behavior;
    d.va = b->process_va ? 1 : 0;
    d.wa = b->process_wa ? 1 : 0;
    d.va_flag = b->va_flag;
    d.swimfast = b->swimfast; d.initsize = b->initsize;
    d.vort_cr = b->vort_cr; d.vort_sat = b->vort_sat; d.b0pv = b->b0pv; d.b1pv = b->b1pv; d.b0wv = b->b0wv;
    d.b1w = b->b1w; d.acc_cr = b->acc_cr; d.acc_sat = b->acc_sat; d.b0pa = b->b0pa; d.b1pa = b->b1pa;
    d.b0wa = b->b0wa;
    const size_t e = (size_t)(ctx->mixed ? 4 : ctx->elem) * RP_SLOTS;   // FP32 in the mixed form
    for (int k = 0; k < ctx->ngrid; k++) {
        GridBuf& G = ctx->g[k];
        const size_t nw = (size_t)G.nx * G.ny * (G.N + 1) * e;
        void** f[4] = {&G.turbaccel, &G.turbvort, &G.waveaccelu, &G.waveaccelv};
        const bool need[4] = {d.va != 0, d.va != 0, d.wa != 0, d.wa != 0};
        for (int q = 0; q < 4; q++) {
            if (!need[q] || *f[q]) continue;
            if (dalloc(f[q], nw)) return fail(ctx, RP_ERR_NOMEM, "rp_set_behavior: field ring allocation");
            CK(cudaMemset(*f[q], 0, nw));
        }
    }
    if ((d.va || d.wa) && !ctx->b_acc) {
        const size_t cap = (size_t)ctx->cap * 8;
        if (dalloc(&ctx->b_acc, cap) || dalloc(&ctx->b_vort, cap) || dalloc(&ctx->b_behavew, cap) ||
            dalloc(&ctx->b_ssf, cap))
            return fail(ctx, RP_ERR_NOMEM, "rp_set_behavior: output allocation");
        CK(cudaMemset(ctx->b_acc, 0, cap));
        CK(cudaMemset(ctx->b_vort, 0, cap));
        CK(cudaMemset(ctx->b_behavew, 0, cap));
        CK(cudaMemset(ctx->b_ssf, 0, cap));
    }
    ctx->beh = d;
    ctx->beh_set = true;
    // HTurb 2, VTurb idt/deltat, then behave's 2 normals and 5 uniforms
    ctx->ndraw = 2 + ctx->prm.idt / (int)ctx->prm.deltat + ((d.va || d.wa) ? 7 : 0);
    return RP_OK;
}

int rp_get_behavior(rp_ctx* ctx, int64_t n, double* acc, double* vort, double* behavew, double* ssf) {
    if (!ctx) return RP_ERR_ARG;
    if (n < 0 || n > ctx->n) return fail(ctx, RP_ERR_ARG, "rp_get_behavior: n exceeds particle count");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->s_comp;
    double* host[4] = {acc, vort, behavew, ssf};
    double* dev[4] = {ctx->b_acc, ctx->b_vort, ctx->b_behavew, ctx->b_ssf};
    for (int c = 0; c < 4; c++) {
        if (!host[c]) continue;
        if (!dev[c]) {                       // no Process_VA / _WA: behout is 0 (behavior_module.f90:226-233)
            std::memset(host[c], 0, (size_t)n * 8);
            continue;
        }
        int rc;
        if (!ctx->permuted) {
            rc = d2h(ctx, host[c], dev[c], (size_t)n * 8, s);
        } else {
            CK(rp::launch_unsort(8, dev[c], ctx->turbv, ctx->pid, ctx->state_base, ctx->n, n, s));
            ctx->launches++;
            rc = d2h(ctx, host[c], ctx->turbv, (size_t)n * 8, s);
        }
        if (rc != RP_OK) return rc;
    }
    return RP_OK;
}

int rp_reset_diagnostics(rp_ctx* ctx) {
    if (!ctx) return RP_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (ctx->n > 0 && (ctx->d_mean_salt || ctx->d_hob)) {
        CK(rp::launch_diag_reset(particles_dev(ctx), ctx->s_comp));
        ctx->launches++;
    }
    return RP_OK;
}

// ------------------------------------------------------------ adjoint pair

int rp_adj_frames(rp_ctx* ctx, int32_t nframes) {
    if (!ctx) return RP_ERR_ARG;
    if (nframes < 3) return fail(ctx, RP_ERR_ARG, "rp_adj_frames: at least 3 frames");
    CK(cudaSetDevice(ctx->device));
    CK(cudaDeviceSynchronize());
    for (int g = 0; g < ctx->ngrid; g++) {
        const GridBuf& G = ctx->g[g];
        const size_t n2 = (size_t)G.nx * G.ny, nu = (size_t)(G.nx - 1) * G.ny, nv = (size_t)G.nx * (G.ny - 1);
        const size_t sz[5] = {n2, nu * G.N, nv * G.N, n2 * (G.N + 1), n2 * (G.N + 1)};
        for (int f = 0; f < 5; f++) {
            if (ctx->adj.fst[g][f]) cudaFree(ctx->adj.fst[g][f]);
            ctx->adj.fst[g][f] = nullptr;
            ctx->adj.fsize[g][f] = sz[f];
            if (dalloc(&ctx->adj.fst[g][f], sz[f] * 8 * (size_t)nframes))
                return fail(ctx, RP_ERR_NOMEM, "rp_adj_frames: frame store allocation");
        }
    }
    ctx->adj.nframes = nframes;
    return RP_OK;
}

int rp_adj_set_frame(rp_ctx* ctx, int32_t ng, int32_t frame, const double* zeta, const double* u, const double* v,
                     const double* w, const double* aks, const double* su, const double* sv) {
    if (!ctx) return RP_ERR_ARG;
    if (ng < 1 || ng > ctx->ngrid) return fail(ctx, RP_ERR_ARG, "rp_adj_set_frame: grid id out of range");
    if (frame < 1 || frame > ctx->adj.nframes)
        return fail(ctx, RP_ERR_ARG, "rp_adj_set_frame: frame out of the store (rp_adj_frames)");
    if (!zeta || !u || !v || !w || !aks) return fail(ctx, RP_ERR_ARG, "rp_adj_set_frame: null field");
    const bool stokes = ctx->prm.stokes != 0;
    if (stokes && (!su || !sv)) return fail(ctx, RP_ERR_ARG, "rp_adj_set_frame: stokes on but su/sv null");
    CK(cudaSetDevice(ctx->device));
    const GridBuf& G = ctx->g[ng - 1];
    auto dst = [&](int f) { return ctx->adj.fst[ng - 1][f] + (size_t)(frame - 1) * ctx->adj.fsize[ng - 1][f]; };
    int rc;
    if ((rc = adj_upload_field(ctx, zeta, nullptr, dst(0), G.nx, G.ny, 1)) ||
        (rc = adj_upload_field(ctx, u, stokes ? su : nullptr, dst(1), G.nx - 1, G.ny, G.N)) ||
        (rc = adj_upload_field(ctx, v, stokes ? sv : nullptr, dst(2), G.nx, G.ny - 1, G.N)) ||
        (rc = adj_upload_field(ctx, w, nullptr, dst(3), G.nx, G.ny, G.N + 1)) ||
        (rc = adj_upload_field(ctx, aks, nullptr, dst(4), G.nx, G.ny, G.N + 1)))
        return rc;
    CK(cudaStreamSynchronize(ctx->s_copy));
    return RP_OK;
}

int rp_forward(rp_ctx* ctx, int32_t nsteps, const rp_adj_step* steps, double kappa, int32_t checkpoint_every) {
    if (!ctx || !steps) return RP_ERR_ARG;
    if (nsteps < 1 || checkpoint_every < 1) return fail(ctx, RP_ERR_ARG, "rp_forward: nsteps, checkpoint_every >= 1");
    if (ctx->adj.nframes < 3) return fail(ctx, RP_ERR_STATE, "rp_forward: load the frame store first");
    if (ctx->permuted) return fail(ctx, RP_ERR_STATE, "rp_forward: particle state is re-sorted; set it again");
    if (ctx->hook) return fail(ctx, RP_ERR_STATE, "rp_forward: the noise hook is not used by the adjoint pair");
    if (ctx->wetdry) return fail(ctx, RP_ERR_UNSUPPORTED, "rp_forward: the adjoint model has the static masks only");
    if (ctx->prm.behavior != 0 || ctx->beh.va || ctx->beh.wa)
        return fail(ctx, RP_ERR_UNSUPPORTED, "rp_forward: the adjoint model is passive (Behavior 0)");
    for (int s = 0; s < nsteps; s++) {
        const rp_adj_step& st = steps[s];
        const int fr[3] = {st.frame_b, st.frame_c, st.frame_f};
        for (int t = 0; t < 3; t++)
            if (fr[t] < 1 || fr[t] > ctx->adj.nframes) return fail(ctx, RP_ERR_ARG, "rp_forward: frame out of the store");
    }
    CK(cudaSetDevice(ctx->device));
    auto& J = ctx->adj;
    const int64_t n = ctx->n;
    const int nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
    const size_t blk = adj_block_bytes(n);
    // (re)allocate for this run
    double* bufs[] = {J.ck, J.prec, J.seg, J.work, J.lx, J.ly, J.lz, J.kbar, J.tan};
    for (double* b : bufs) if (b) cudaFree(b);
    J.ck = J.prec = J.seg = J.work = J.lx = J.ly = J.lz = J.kbar = J.tan = nullptr;
    if (dalloc(&J.ck, blk * (size_t)(nseg + 1)) || dalloc(&J.prec, (size_t)nsteps * n * 8) ||
        dalloc(&J.seg, blk * (size_t)checkpoint_every) || dalloc(&J.work, blk) || dalloc(&J.lx, (size_t)n * 8) ||
        dalloc(&J.ly, (size_t)n * 8) || dalloc(&J.lz, (size_t)n * 8) || dalloc(&J.kbar, (size_t)n * 8) ||
        dalloc(&J.tan, (size_t)n * 12 * 8))
        return fail(ctx, RP_ERR_NOMEM, "rp_forward: checkpoint / record allocation");
    J.steps.assign(steps, steps + nsteps);
    J.ckpt = checkpoint_every;
    J.n = n;
    J.kappa = kappa;
    cudaStream_t s = ctx->s_comp;
    const rp::AdjStateDev cur = adj_ctx_state(ctx);
    for (int k = 0; k < nsteps; k++) {
        if (k % checkpoint_every == 0)
            CK(adj_copy(cur, adj_view((char*)J.ck + blk * (size_t)(k / checkpoint_every), n), n, s));
        RpStepArgs A;
        AdjFrames F;
        adj_args(ctx, J.steps[k], A, F, n);
        CK(rp::launch_adj(0, A, F, cur, J.prec + (size_t)k * n, 1, kappa, nullptr, nullptr, nullptr, nullptr, nullptr,
                          ctx->npmax, s, ctx->num_sms));
        ctx->launches++;
    }
    CK(adj_copy(cur, adj_view((char*)J.ck + blk * (size_t)nseg, n), n, s));   // final state
    CK(cudaStreamSynchronize(s));
    return RP_OK;
}

int rp_backward(rp_ctx* ctx, const double* dL_dx, const double* dL_dy, const double* dL_dz, double* dL_dx0,
                double* dL_dy0, double* dL_dz0, double* dL_dkappa) {
    if (!ctx || !dL_dx || !dL_dy || !dL_dz) return RP_ERR_ARG;
    auto& J = ctx->adj;
    if (J.steps.empty() || !J.ck) return fail(ctx, RP_ERR_STATE, "rp_backward: call rp_forward first");
    CK(cudaSetDevice(ctx->device));
    const int64_t n = J.n;
    const int nsteps = (int)J.steps.size();
    const size_t blk = adj_block_bytes(n);
    cudaStream_t s = ctx->s_comp;
    int rc;
    if ((rc = h2d(ctx, J.lx, dL_dx, (size_t)n * 8, s)) || (rc = h2d(ctx, J.ly, dL_dy, (size_t)n * 8, s)) ||
        (rc = h2d(ctx, J.lz, dL_dz, (size_t)n * 8, s)))
        return rc;
    CK(cudaMemsetAsync(J.kbar, 0, (size_t)n * 8, s));
    const int nseg = (nsteps + J.ckpt - 1) / J.ckpt;
    const rp::AdjStateDev work = adj_view(J.work, n);
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int k0 = sg * J.ckpt, k1 = std::min(nsteps, k0 + J.ckpt);
        // recompute the segment's step-start states from its checkpoint
        CK(adj_copy(adj_view((char*)J.ck + blk * (size_t)sg, n), work, n, s));
        for (int k = k0; k < k1; k++) {
            CK(adj_copy(work, adj_view((char*)J.seg + blk * (size_t)(k - k0), n), n, s));
            if (k + 1 < k1) {
                RpStepArgs A;
                AdjFrames F;
                adj_args(ctx, J.steps[k], A, F, n);
                CK(rp::launch_adj(0, A, F, work, J.prec + (size_t)k * n, 0, J.kappa, nullptr, nullptr, nullptr, nullptr,
                                  nullptr, ctx->npmax, s, ctx->num_sms));
                ctx->launches++;
            }
        }
        // reverse steps of the segment
        for (int k = k1 - 1; k >= k0; k--) {
            RpStepArgs A;
            AdjFrames F;
            adj_args(ctx, J.steps[k], A, F, n);
            CK(rp::launch_adj(2, A, F, adj_view((char*)J.seg + blk * (size_t)(k - k0), n), J.prec + (size_t)k * n, 0,
                              J.kappa, nullptr, J.lx, J.ly, J.lz, J.kbar, ctx->npmax, s, ctx->num_sms));
            ctx->launches++;
        }
    }
    if ((dL_dx0 && (rc = d2h(ctx, dL_dx0, J.lx, (size_t)n * 8, s))) ||
        (dL_dy0 && (rc = d2h(ctx, dL_dy0, J.ly, (size_t)n * 8, s))) ||
        (dL_dz0 && (rc = d2h(ctx, dL_dz0, J.lz, (size_t)n * 8, s))))
        return rc;
    if (dL_dkappa) {
        std::vector<double> kb((size_t)n);
        if ((rc = d2h(ctx, kb.data(), J.kbar, (size_t)n * 8, s))) return rc;
        double acc = 0.0;
        for (double v : kb) acc += v;
        *dL_dkappa = acc;
    }
    return RP_OK;
}

int rp_adj_replay(rp_ctx* ctx, const double* x0, const double* y0, const double* z0, double kappa, double* xf,
                  double* yf, double* zf) {
    if (!ctx) return RP_ERR_ARG;
    auto& J = ctx->adj;
    if (J.steps.empty() || !J.ck) return fail(ctx, RP_ERR_STATE, "rp_adj_replay: call rp_forward first");
    CK(cudaSetDevice(ctx->device));
    const int64_t n = J.n;
    cudaStream_t s = ctx->s_comp;
    const rp::AdjStateDev work = adj_view(J.work, n);
    CK(adj_copy(adj_view(J.ck, n), work, n, s));
    int rc;
    if ((x0 && (rc = h2d(ctx, work.x, x0, (size_t)n * 8, s))) || (y0 && (rc = h2d(ctx, work.y, y0, (size_t)n * 8, s))) ||
        (z0 && (rc = h2d(ctx, work.z, z0, (size_t)n * 8, s))))
        return rc;
    for (size_t k = 0; k < J.steps.size(); k++) {
        RpStepArgs A;
        AdjFrames F;
        adj_args(ctx, J.steps[k], A, F, n);
        CK(rp::launch_adj(0, A, F, work, J.prec + k * n, 0, kappa, nullptr, nullptr, nullptr, nullptr, nullptr,
                          ctx->npmax, s, ctx->num_sms));
        ctx->launches++;
    }
    if ((xf && (rc = d2h(ctx, xf, work.x, (size_t)n * 8, s))) || (yf && (rc = d2h(ctx, yf, work.y, (size_t)n * 8, s))) ||
        (zf && (rc = d2h(ctx, zf, work.z, (size_t)n * 8, s))))
        return rc;
    return RP_OK;
}

int rp_tangent(rp_ctx* ctx, double kappa, double* jac) {
    if (!ctx || !jac) return RP_ERR_ARG;
    auto& J = ctx->adj;
    if (J.steps.empty() || !J.ck) return fail(ctx, RP_ERR_STATE, "rp_tangent: call rp_forward first");
    CK(cudaSetDevice(ctx->device));
    const int64_t n = J.n;
    cudaStream_t s = ctx->s_comp;
    const rp::AdjStateDev work = adj_view(J.work, n);
    CK(adj_copy(adj_view(J.ck, n), work, n, s));
    CK(rp::launch_adj_tangent_init(J.tan, n, s));
    for (size_t k = 0; k < J.steps.size(); k++) {
        RpStepArgs A;
        AdjFrames F;
        adj_args(ctx, J.steps[k], A, F, n);
        CK(rp::launch_adj(1, A, F, work, J.prec + k * n, 0, kappa, J.tan, nullptr, nullptr, nullptr, nullptr,
                          ctx->npmax, s, ctx->num_sms));
        ctx->launches++;
    }
    return d2h(ctx, jac, J.tan, (size_t)n * 12 * 8, s);
}

int rp_set_launch(rp_ctx* ctx, int32_t resort, int32_t blocks_per_sm) {
    if (!ctx) return RP_ERR_ARG;
    if (resort < 0 || blocks_per_sm < 0) return fail(ctx, RP_ERR_ARG, "rp_set_launch: values must be >= 0");
    CK(cudaSetDevice(ctx->device));
    if (resort > 0) {
        CK(cudaStreamSynchronize(ctx->s_comp));
        const int rc = sort_buffers(ctx);
        if (rc != RP_OK) return rc;
    }
    ctx->resort = resort;
    ctx->prm.reserved[1] = resort;
    ctx->prm.reserved[2] = blocks_per_sm;
    if (ctx->since_sort > resort) ctx->since_sort = resort;
    return RP_OK;
}

int rp_set_kernel_form(rp_ctx* ctx, int32_t form) {
    if (!ctx) return RP_ERR_ARG;
    if (form < 0 || form > 5) return fail(ctx, RP_ERR_ARG, "rp_set_kernel_form: form must be 0..5");
    ctx->prm.reserved[0] = form;
    return RP_OK;
}

int rp_set_id_base(rp_ctx* ctx, uint32_t base) {
    if (!ctx) return RP_ERR_ARG;
    ctx->pid_base = base;
    return RP_OK;
}

int rp_set_step_index(rp_ctx* ctx, uint64_t step_index) {
    if (!ctx) return RP_ERR_ARG;
    ctx->step_index = step_index;
    return RP_OK;
}

int rp_set_noise_hook(rp_ctx* ctx, const double* noise, int64_t nsteps) {
    if (!ctx) return RP_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (ctx->hook) {
        CK(cudaStreamSynchronize(ctx->s_comp));
        cudaFree(ctx->hook);
        ctx->hook = nullptr;
    }
    ctx->hook_steps = 0;
    ctx->hook_pos = 0;
    if (!noise) return RP_OK;
    if (nsteps <= 0 || ctx->n <= 0) return fail(ctx, RP_ERR_ARG, "rp_set_noise_hook: set particles first, nsteps > 0");
    const size_t bytes = (size_t)nsteps * ctx->n * ctx->ndraw * 8;
    CK(cudaMalloc(&ctx->hook, bytes));
    int rc = h2d(ctx, ctx->hook, noise, bytes, ctx->s_comp);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->s_comp));
    ctx->hook_steps = nsteps;
    return RP_OK;
}

int rp_synchronize(rp_ctx* ctx) {
    if (!ctx) return RP_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->s_copy));
    CK(cudaStreamSynchronize(ctx->s_comp));
    CK(cudaStreamSynchronize(ctx->s_out));
    ctx->out_pending = false;
    return RP_OK;
}

int rp_device_state_get(rp_ctx* ctx, rp_device_state* out) {
    if (!ctx || !out) return RP_ERR_ARG;
    if (ctx->mixed && ctx->n > 0) {
        CK(cudaSetDevice(ctx->device));
        CK(rp::launch_mixed_convert(particles_dev(ctx), 1, ctx->s_comp));
        ctx->launches++;
        CK(cudaStreamSynchronize(ctx->s_comp));
    }
    out->n = ctx->n;
    out->x = ctx->x; out->y = ctx->y; out->z = ctx->z; out->age = ctx->age; out->dob = ctx->dob;
    out->status = ctx->status; out->wd = ctx->wd; out->zeta = ctx->zeta; out->bath = ctx->bath;
    out->gid = ctx->gid; out->isin = ctx->isin; out->pid = ctx->pid; out->flags = ctx->flags;
    out->stream = (void*)ctx->s_comp;
    return RP_OK;
}

int rp_kernel_launches(rp_ctx* ctx, int64_t* count) {
    if (!ctx || !count) return RP_ERR_ARG;
    *count = ctx->launches;
    return RP_OK;
}

int rp_count_spline_passes(rp_ctx* ctx, int32_t on) {
    if (!ctx) return RP_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (on && !ctx->d_spl) CK(cudaMalloc(&ctx->d_spl, 2 * sizeof(unsigned long long)));
    if (on) CK(cudaMemsetAsync(ctx->d_spl, 0, 2 * sizeof(unsigned long long), ctx->s_comp));
    ctx->spl_on = on != 0;
    return RP_OK;
}

int rp_spline_pass_counts(rp_ctx* ctx, int64_t* fits, int64_t* passes) {
    if (!ctx) return RP_ERR_ARG;
    if (!ctx->d_spl) return fail(ctx, RP_ERR_STATE, "rp_spline_pass_counts: counting was never started");
    cudaSetDevice(ctx->device);
    unsigned long long h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, ctx->d_spl, sizeof h, cudaMemcpyDeviceToHost, ctx->s_comp));
    CK(cudaStreamSynchronize(ctx->s_comp));
    if (fits) *fits = (int64_t)h[0];
    if (passes) *passes = (int64_t)h[1];
    return RP_OK;
}

int rp_last_step_stats(rp_ctx* ctx, float* ms, int32_t* kernels) {
    if (!ctx) return RP_ERR_ARG;
    if (!ctx->timed) return fail(ctx, RP_ERR_STATE, "no step launched yet");
    CK(cudaEventSynchronize(ctx->ev1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    if (ms) *ms = t;
    if (kernels) *kernels = ctx->last_kernels;
    return RP_OK;
}

}  // extern "C"
