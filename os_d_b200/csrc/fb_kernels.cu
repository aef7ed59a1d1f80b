// fb_kernels.cu -- f-basis Lindblad RK4 on the GPU (density-matrix oracle of the QJ ensemble).
//
// The reference integrates dx/dt = Gs x + E(t) Qs_drv x - Ks with classic RK4
// (source/cpp/CQdiss_os_dimer/CQdiss/calcODE.cpp:75-118 calcVectValue_real, :249-389
// calcODE_trans/std), two mkl_dcsrgemv per stage.  Two GPU paths:
//   * rk4_cluster: one thread-block cluster holds the whole system in distributed shared memory
//     and integrates a period per launch (systems that fit <= 16 CTAs);
//   * rk_stage: one launch per RK stage (four per step) computes both CSR row products, the
//     stage vector k = (Gs x + drv Qs x - Ks) h and the next stage argument, or in stage 4 the
//     RK4 update of x.  The stage arguments are double-buffered (stage s reads one buffer and
//     writes the other), as the reference keeps x, tmp and k1..k4 apart (calcODE.cpp:249-309):
//     a row may read any other row's argument, and rows of one launch run in no fixed order.
//
// Canonical row sum (shared bit-for-bit with the CPU oracle): lane l of a warp accumulates
// the row's nonzeros l, l+32, l+64, ... in CSR order with fma, then the 32 partial sums are
// combined by an xor butterfly (offsets 16, 8, 4, 2, 1).  All other arithmetic is literal
// (-fmad=false).  The drive uses sin() of the stage time (CUDA libdevice), so drv_type 1
// matches the CPU within rounding, not bit-for-bit.
#include <cooperative_groups.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/qjx_b200.h"

namespace fb {

struct FbParams {
    int n;
    const int *gr, *gc;
    const double *gv;
    const int *qr, *qc;
    const double *qv;
    const double *Ks;
    double drv_ampl;  // -A (calcODE.cpp:91)
    double drv_freq, drv_phase;
    int drv_type;
    double *x;
    double *va, *vb;     // stage arguments: stage 1 writes va, 2 writes vb, 3 writes va
    double *k1, *k2, *k3;
};

__device__ __forceinline__ double warp_row_sum(const int *rp, const int *ci, const double *v, const double *x, int row,
                                               int lane)
{
    double s = 0.0;
    const int b = rp[row], e = rp[row + 1];
    for (int j = b + lane; j < e; j += 32) s = __fma_rn(v[j], x[ci[j]], s);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, off));
    return s;
}

// Stage 1..4 of one RK4 step at time t (calcODE.cpp:278-302), one warp per row.  Stage s reads
// its argument (x, va, vb, va) and writes only a buffer no row of this launch reads (va, vb, va,
// and in stage 4 the row's own x: x += (k1 + 2 k2 + 2 k3 + k4) / 6, calcODE.cpp:299-302).
__global__ void rk_stage(const FbParams P, int stage, double t, double h)
{
    const int warps = blockDim.x >> 5;
    const int row = blockIdx.x * warps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= P.n) return;
    const double *arg = (stage == 1) ? P.x : ((stage == 3) ? P.vb : P.va);
    const double tt = (stage == 1) ? t : ((stage == 4) ? __dadd_rn(t, h) : __dadd_rn(t, __ddiv_rn(h, 2.0)));
    const double t1 = warp_row_sum(P.gr, P.gc, P.gv, arg, row, lane);
    const double t2 = warp_row_sum(P.qr, P.qc, P.qv, arg, row, lane);
    if (lane != 0) return;
    double drv;
    const double sn = sin(__dadd_rn(__dmul_rn(P.drv_freq, tt), P.drv_phase));
    if (P.drv_type == 1) drv = __dmul_rn(P.drv_ampl, sn);
    else drv = __dmul_rn(P.drv_ampl, (sn < 0.0) ? -1.0 : 1.0);
    const double k = __dmul_rn(__dsub_rn(__dadd_rn(t1, __dmul_rn(drv, t2)), P.Ks[row]), h);
    const double x = P.x[row];
    if (stage == 1) {
        P.k1[row] = k;
        P.va[row] = __dadd_rn(x, __ddiv_rn(k, 2.0));
    } else if (stage == 2) {
        P.k2[row] = k;
        P.vb[row] = __dadd_rn(x, __ddiv_rn(k, 2.0));
    } else if (stage == 3) {
        P.k3[row] = k;
        P.va[row] = __dadd_rn(x, k);
    } else {
        const double sum =
            __dadd_rn(__dadd_rn(__dadd_rn(P.k1[row], __dmul_rn(2.0, P.k2[row])), __dmul_rn(2.0, P.k3[row])), k);
        P.x[row] = __dadd_rn(x, __ddiv_rn(sum, 6.0));
    }
}

// Queues the four stage launches of every RK4 step of n_periods periods from period0 on `st`;
// returns the first launch error (cudaLaunchKernelEx reports the launch's own status).
static cudaError_t queue_rk_stages(const FbParams &P, double T, int num_steps, int period0, int n_periods,
                                   cudaStream_t st)
{
    const double step = T / double(num_steps);  // data.cpp:10
    const int warps = 8;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((P.n + warps - 1) / warps);
    lc.blockDim = dim3(warps * 32);
    lc.stream = st;
    for (int p = period0; p < period0 + n_periods; p++)
        for (int s = 0; s < num_steps; s++) {
            const double t = double(p) * T + double(s) * step;  // calcODE.cpp:280
            for (int stage = 1; stage <= 4; stage++) {
                const cudaError_t e = cudaLaunchKernelEx(&lc, rk_stage, P, stage, t, step);
                if (e != cudaSuccess) return e;
            }
        }
    return cudaSuccess;
}

// ---------------------------------------------------------------- cluster-resident RK4
// One thread-block cluster integrates the whole system: CTA r owns rows [row_lo[r], row_lo[r+1])
// and keeps their CSR slices of Gs and Qs_drv in shared memory (the cluster's distributed shared
// memory holds the whole Liouvillian), plus full copies of x and of the two stage arguments.
// Each stage computes the owned rows and stores the next stage argument into every CTA of the
// cluster (DSMEM); a hardware cluster barrier separates the stages, four per RK4 step, and no
// kernel launch happens inside a period.  Rows are computed thread-per-row with the canonical
// 32-lane order (lane partial sums over nonzeros l, l+32, ..., then the butterfly tree), so the
// results equal the warp-per-row kernel bit for bit.
struct FbClusterParams {
    int n;
    const int *row_lo;  // [cluster size + 1]
    const int *gr, *gc;
    const double *gv;
    const int *qr, *qc;
    const double *qv;
    const double *Ks;
    double *x;
    double drv_ampl, drv_freq, drv_phase;
    int drv_type;
    double T, h;
    int num_steps, period0, n_periods;
    int max_rows, max_gnz, max_qnz;
};

__device__ __forceinline__ double row_sum_lanes(const int *rp, const int *col, const double *val, const double *arg,
                                                int r)
{
    const int b = rp[r], e = rp[r + 1];
    // A row with at most one nonzero (every row of the drive matrix Qs, so warps do not diverge
    // here): lane 0 holds fma(v, a, 0) and the tree adds only +0.0 to it, which leaves every value
    // but -0 unchanged and turns -0 into +0, i.e. the result is p0 + 0.0.
    if (e - b <= 1) return e > b ? __dadd_rn(__fma_rn(val[b], arg[col[b]], 0.0), 0.0) : 0.0;
    double p[32];
#pragma unroll
    for (int l = 0; l < 32; l++) p[l] = 0.0;
    for (int base = b; base < e; base += 32) {
#pragma unroll
        for (int l = 0; l < 32; l++) {
            const int j = base + l;
            if (j < e) p[l] = __fma_rn(val[j], arg[col[j]], p[l]);
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
        for (int l = 0; l < off; l++) p[l] = __dadd_rn(p[l], p[l + off]);
    return p[0];
}

constexpr int kMaxCluster = 16;

__global__ void __launch_bounds__(512, 1) rk4_cluster(const FbClusterParams P)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), cs = (int)cl.num_blocks();
    extern __shared__ __align__(16) unsigned char fsm[];
    const int n = P.n, tid = threadIdx.x, nt = blockDim.x;
    double *xf = reinterpret_cast<double *>(fsm);
    double *va = xf + n;
    double *vb = va + n;
    double *k1 = vb + n;
    double *k2 = k1 + P.max_rows;
    double *k3 = k2 + P.max_rows;
    double *ks = k3 + P.max_rows;
    double *gval = ks + P.max_rows;
    double *qval = gval + P.max_gnz;
    int *grp = reinterpret_cast<int *>(qval + P.max_qnz);
    int *qrp = grp + P.max_rows + 1;
    int *gcol = qrp + P.max_rows + 1;
    int *qcol = gcol + P.max_gnz;
    const int r0 = P.row_lo[rank], nr = P.row_lo[rank + 1] - r0;
    const int gb = P.gr[r0], qb = P.qr[r0];
    for (int i = tid; i < n; i += nt) xf[i] = P.x[i];
    for (int i = tid; i <= nr; i += nt) {
        grp[i] = P.gr[r0 + i] - gb;
        qrp[i] = P.qr[r0 + i] - qb;
    }
    for (int j = tid; j < P.gr[r0 + nr] - gb; j += nt) {
        gval[j] = P.gv[gb + j];
        gcol[j] = P.gc[gb + j];
    }
    for (int j = tid; j < P.qr[r0 + nr] - qb; j += nt) {
        qval[j] = P.qv[qb + j];
        qcol[j] = P.qc[qb + j];
    }
    for (int i = tid; i < nr; i += nt) ks[i] = P.Ks[r0 + i];
    cl.sync();
    const double h = P.h;
    for (int p = P.period0; p < P.period0 + P.n_periods; p++) {
        for (int s = 0; s < P.num_steps; s++) {
            const double t = __dadd_rn(__dmul_rn((double)p, P.T), __dmul_rn((double)s, h));
#pragma unroll 1
            for (int stage = 1; stage <= 4; stage++) {
                const double *arg = (stage == 1) ? xf : ((stage == 3) ? vb : va);
                const double tt =
                    (stage == 1) ? t : ((stage == 4) ? __dadd_rn(t, h) : __dadd_rn(t, __ddiv_rn(h, 2.0)));
                const double sn = sin(__dadd_rn(__dmul_rn(P.drv_freq, tt), P.drv_phase));
                const double drv = (P.drv_type == 1) ? __dmul_rn(P.drv_ampl, sn)
                                                     : __dmul_rn(P.drv_ampl, (sn < 0.0) ? -1.0 : 1.0);
                for (int i = tid; i < nr; i += nt) {
                    const double t1 = row_sum_lanes(grp, gcol, gval, arg, i);
                    const double t2 = row_sum_lanes(qrp, qcol, qval, arg, i);
                    const double k = __dmul_rn(__dsub_rn(__dadd_rn(t1, __dmul_rn(drv, t2)), ks[i]), h);
                    const int row = r0 + i;
                    const double x = xf[row];
                    if (stage == 1) {
                        k1[i] = k;
                        const double v = __dadd_rn(x, __ddiv_rn(k, 2.0));
                        for (int r = 0; r < cs; r++) *cl.map_shared_rank(va + row, r) = v;
                    } else if (stage == 2) {
                        k2[i] = k;
                        const double v = __dadd_rn(x, __ddiv_rn(k, 2.0));
                        for (int r = 0; r < cs; r++) *cl.map_shared_rank(vb + row, r) = v;
                    } else if (stage == 3) {
                        k3[i] = k;
                        const double v = __dadd_rn(x, k);
                        for (int r = 0; r < cs; r++) *cl.map_shared_rank(va + row, r) = v;
                    } else {
                        const double sum =
                            __dadd_rn(__dadd_rn(__dadd_rn(k1[i], __dmul_rn(2.0, k2[i])), __dmul_rn(2.0, k3[i])), k);
                        const double xn = __dadd_rn(x, __ddiv_rn(sum, 6.0));
                        for (int r = 0; r < cs; r++) *cl.map_shared_rank(xf + row, r) = xn;
                    }
                }
                cl.sync();
            }
        }
    }
    for (int i = tid; i < nr; i += nt) P.x[r0 + i] = xf[r0 + i];
}

}  // namespace fb

struct qjx_fb {
    fb::FbParams P{};
    // cluster-resident path (used when the system fits the shared memory of <= 16 CTAs)
    bool cluster = false;
    int cs = 0;
    size_t csmem = 0;
    fb::FbClusterParams CP{};
    int device = 0;
    double T = 0.0;
    int num_steps = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<void *> allocs;
    double last_ms = 0.0;
};

static void *fb_alloc(qjx_fb *h, size_t bytes)
{
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
    h->allocs.push_back(p);
    return p;
}

extern "C" qjx_status qjx_fb_create(int n, const int *gs_rowptr, const int *gs_col, const double *gs_val,
                                    const int *qs_rowptr, const int *qs_col, const double *qs_val, const double *Ks,
                                    const double *x0, double drv_ampl, double drv_freq, double drv_phase, int drv_type,
                                    double T, int num_steps, int device, qjx_fb **out)
{
    if (n < 1 || !gs_rowptr || !gs_col || !gs_val || !qs_rowptr || !qs_col || !qs_val || !Ks || !x0 || !out ||
        num_steps < 1 || !(T > 0.0) || (drv_type != 0 && drv_type != 1))
        return QJX_ERR_INVALID_ARG;
    *out = nullptr;
    qjx_fb *h = new (std::nothrow) qjx_fb();
    if (!h) return QJX_ERR_OOM;
    h->device = device;
    h->T = T;
    h->num_steps = num_steps;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete h;
        return QJX_ERR_CUDA;
    }
    cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    cudaEventCreate(&h->e0);
    cudaEventCreate(&h->e1);
    const int gnz = gs_rowptr[n], qnz = qs_rowptr[n];
    fb::FbParams &P = h->P;
    P.n = n;
    int *gr = (int *)fb_alloc(h, sizeof(int) * (n + 1)), *gc = (int *)fb_alloc(h, sizeof(int) * gnz);
    int *qr = (int *)fb_alloc(h, sizeof(int) * (n + 1)), *qc = (int *)fb_alloc(h, sizeof(int) * qnz);
    double *gv = (double *)fb_alloc(h, sizeof(double) * gnz), *qv = (double *)fb_alloc(h, sizeof(double) * qnz);
    double *ks = (double *)fb_alloc(h, sizeof(double) * n);
    P.x = (double *)fb_alloc(h, sizeof(double) * n);
    P.va = (double *)fb_alloc(h, sizeof(double) * n);
    P.vb = (double *)fb_alloc(h, sizeof(double) * n);
    P.k1 = (double *)fb_alloc(h, sizeof(double) * n);
    P.k2 = (double *)fb_alloc(h, sizeof(double) * n);
    P.k3 = (double *)fb_alloc(h, sizeof(double) * n);
    if (!gr || !gc || !qr || !qc || !gv || !qv || !ks || !P.x || !P.va || !P.vb || !P.k1 || !P.k2 || !P.k3) {
        qjx_fb_destroy(h);
        return QJX_ERR_OOM;
    }
    cudaMemcpy(gr, gs_rowptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(gc, gs_col, sizeof(int) * gnz, cudaMemcpyHostToDevice);
    cudaMemcpy(gv, gs_val, sizeof(double) * gnz, cudaMemcpyHostToDevice);
    cudaMemcpy(qr, qs_rowptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(qc, qs_col, sizeof(int) * qnz, cudaMemcpyHostToDevice);
    cudaMemcpy(qv, qs_val, sizeof(double) * qnz, cudaMemcpyHostToDevice);
    cudaMemcpy(ks, Ks, sizeof(double) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(P.x, x0, sizeof(double) * n, cudaMemcpyHostToDevice);
    P.gr = gr;
    P.gc = gc;
    P.gv = gv;
    P.qr = qr;
    P.qc = qc;
    P.qv = qv;
    P.Ks = ks;
    P.drv_ampl = -drv_ampl;
    P.drv_freq = drv_freq;
    P.drv_phase = drv_phase;
    P.drv_type = drv_type;
    if (cudaDeviceSynchronize() != cudaSuccess) {
        qjx_fb_destroy(h);
        return QJX_ERR_CUDA;
    }
    // cluster-resident path: smallest cluster (power of two <= 16) whose CTAs hold their rows'
    // CSR slices plus three full vectors in shared memory; QJX_FB_PATH=stages forces the
    // per-stage kernels.
    const char *path = std::getenv("QJX_FB_PATH");
    const bool stages_only = path && std::string(path) == "stages";
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    for (int cs = 1; cs <= fb::kMaxCluster && !stages_only && !h->cluster; cs *= 2) {
        // balanced contiguous row split by nonzeros + a fixed cost per row
        std::vector<int> lo(cs + 1, n);
        lo[0] = 0;
        const long long total = (long long)gnz + qnz + 8LL * n;
        int r = 0;
        long long acc = 0;
        for (int c = 1; c < cs; c++) {
            const long long target = total * c / cs;
            while (r < n && acc + (gs_rowptr[r + 1] - gs_rowptr[r]) + (qs_rowptr[r + 1] - qs_rowptr[r]) + 8 <= target) {
                acc += (gs_rowptr[r + 1] - gs_rowptr[r]) + (qs_rowptr[r + 1] - qs_rowptr[r]) + 8;
                r++;
            }
            lo[c] = r;
        }
        int mr = 0, mg = 0, mq = 0;
        for (int c = 0; c < cs; c++) {
            mr = std::max(mr, lo[c + 1] - lo[c]);
            mg = std::max(mg, gs_rowptr[lo[c + 1]] - gs_rowptr[lo[c]]);
            mq = std::max(mq, qs_rowptr[lo[c + 1]] - qs_rowptr[lo[c]]);
        }
        const size_t bytes = sizeof(double) * (3 * (size_t)n + 4 * (size_t)mr + mg + mq) +
                             sizeof(int) * (2 * (size_t)(mr + 1) + mg + mq);
        if (bytes + 1024 > (size_t)smem_optin) continue;
        if (cudaFuncSetAttribute(fb::rk4_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
            continue;
        if (cs > 8 && cudaFuncSetAttribute(fb::rk4_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
            continue;
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(cs);
        lc.blockDim = dim3(512);
        lc.dynamicSmemBytes = bytes;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, fb::rk4_cluster, &lc) != cudaSuccess || nclusters < 1) {
            cudaGetLastError();
            continue;
        }
        int *d_lo = (int *)fb_alloc(h, sizeof(int) * (cs + 1));
        if (!d_lo) break;
        cudaMemcpy(d_lo, lo.data(), sizeof(int) * (cs + 1), cudaMemcpyHostToDevice);
        fb::FbClusterParams &C = h->CP;
        C.n = n;
        C.row_lo = d_lo;
        C.gr = P.gr;
        C.gc = P.gc;
        C.gv = P.gv;
        C.qr = P.qr;
        C.qc = P.qc;
        C.qv = P.qv;
        C.Ks = P.Ks;
        C.x = P.x;
        C.drv_ampl = P.drv_ampl;
        C.drv_freq = P.drv_freq;
        C.drv_phase = P.drv_phase;
        C.drv_type = P.drv_type;
        C.T = T;
        C.h = T / double(num_steps);
        C.num_steps = num_steps;
        C.max_rows = mr;
        C.max_gnz = mg;
        C.max_qnz = mq;
        h->cluster = true;
        h->cs = cs;
        h->csmem = bytes;
    }
    cudaGetLastError();
    *out = h;
    return QJX_OK;
}

extern "C" qjx_status qjx_fb_run(qjx_fb *h, int period0, int n_periods)
{
    if (!h || period0 < 0 || n_periods < 0) return QJX_ERR_INVALID_ARG;
    if (cudaSetDevice(h->device) != cudaSuccess) return QJX_ERR_CUDA;
    const fb::FbParams &P = h->P;
    cudaEventRecord(h->e0, h->stream);
    if (h->cluster) {  // one cluster launch per period
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(h->cs);
        lc.blockDim = dim3(512);
        lc.dynamicSmemBytes = h->csmem;
        lc.stream = h->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = h->cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        for (int p = period0; p < period0 + n_periods; p++) {
            fb::FbClusterParams C = h->CP;
            C.period0 = p;
            C.n_periods = 1;
            if (cudaLaunchKernelEx(&lc, fb::rk4_cluster, C) != cudaSuccess) return QJX_ERR_CUDA;
        }
    } else if (fb::queue_rk_stages(P, h->T, h->num_steps, period0, n_periods, h->stream) != cudaSuccess) {
        return QJX_ERR_CUDA;
    }
    cudaEventRecord(h->e1, h->stream);
    if (cudaEventSynchronize(h->e1) != cudaSuccess) return QJX_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->e0, h->e1);
    h->last_ms = ms;
    return QJX_OK;
}

extern "C" qjx_status qjx_fb_info(qjx_fb *h, int *cluster_size)
{
    if (!h || !cluster_size) return QJX_ERR_INVALID_ARG;
    *cluster_size = h->cluster ? h->cs : 0;
    return QJX_OK;
}

extern "C" qjx_status qjx_fb_get(qjx_fb *h, double *x, double *last_period_ms)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    if (cudaSetDevice(h->device) != cudaSuccess) return QJX_ERR_CUDA;
    if (x && cudaMemcpy(x, h->P.x, sizeof(double) * h->P.n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return QJX_ERR_CUDA;
    if (last_period_ms) *last_period_ms = h->last_ms;
    return QJX_OK;
}

// ---------------------------------------------------------------- allocation-free variant
// Stage vectors va, vb, k1, k2, k3 of the allocation-free entry point, one static array shared by
// all its calls on a device.  In host code this name is only a stand-in for the symbol; its
// device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_fb_noalloc_scratch[5 * QJX_FB_NOALLOC_MAX_N];

static double *fb_noalloc_scratch_ptr(int device)
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static double *ptr[kMaxDevices] = {nullptr};
    if (device < 0 || device >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_fb_noalloc_scratch) != cudaSuccess) return nullptr;
        ptr[device] = static_cast<double *>(p);
    }
    return ptr[device];
}

extern "C" qjx_status qjx_fb_rk4_noalloc(int n, const int *gs_rowptr, const int *gs_col, const double *gs_val,
                                         const int *qs_rowptr, const int *qs_col, const double *qs_val,
                                         const double *Ks, double *x, double drv_ampl, double drv_freq,
                                         double drv_phase, int drv_type, double T, int num_steps, int period0,
                                         int n_periods, int device, void *stream)
{
    if (n < 1 || !gs_rowptr || !gs_col || !gs_val || !qs_rowptr || !qs_col || !qs_val || !Ks || !x ||
        num_steps < 1 || !(T > 0.0) || (drv_type != 0 && drv_type != 1) || period0 < 0 || n_periods < 0)
        return QJX_ERR_INVALID_ARG;
    if (n > QJX_FB_NOALLOC_MAX_N) return QJX_ERR_UNSUPPORTED;
    if (cudaSetDevice(device) != cudaSuccess) return QJX_ERR_CUDA;
    double *scratch = fb_noalloc_scratch_ptr(device);
    if (!scratch) return QJX_ERR_CUDA;
    fb::FbParams P{};
    P.n = n;
    P.gr = gs_rowptr;
    P.gc = gs_col;
    P.gv = gs_val;
    P.qr = qs_rowptr;
    P.qc = qs_col;
    P.qv = qs_val;
    P.Ks = Ks;
    P.drv_ampl = -drv_ampl;
    P.drv_freq = drv_freq;
    P.drv_phase = drv_phase;
    P.drv_type = drv_type;
    P.x = x;
    P.va = scratch;
    P.vb = scratch + QJX_FB_NOALLOC_MAX_N;
    P.k1 = scratch + 2 * QJX_FB_NOALLOC_MAX_N;
    P.k2 = scratch + 3 * QJX_FB_NOALLOC_MAX_N;
    P.k3 = scratch + 4 * QJX_FB_NOALLOC_MAX_N;
    // only the status of this call's own launches is reported; an error left by other code
    // stays where the caller can still read it
    const cudaError_t e =
        fb::queue_rk_stages(P, T, num_steps, period0, n_periods, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? QJX_OK : QJX_ERR_CUDA;
}

extern "C" void qjx_fb_destroy(qjx_fb *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void *p : h->allocs) cudaFree(p);
    if (h->e0) cudaEventDestroy(h->e0);
    if (h->e1) cudaEventDestroy(h->e1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}
