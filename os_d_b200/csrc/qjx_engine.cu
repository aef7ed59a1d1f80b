// qjx_engine.cu -- host side of the QJ trajectory engine: device memory, the micro-step
// loop (CUDA graphs of 6 micro-steps, bounded host polling), jump-record draining, and the
// C ABI declared in include/qjx_b200.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>
#include <sys/stat.h>

#include "../../include/qjx_b200.h"
#include "qjx_device.cuh"

namespace qjx {
cudaError_t launch_step(const Params &P, int s, int grid, cudaStream_t st);
cudaError_t launch_split_steps(const Params &P, int s0, int nsteps, int grid, cudaStream_t st);
int pick_layout(int d, int *rows_per_block);
cudaError_t launch_dmma_peak(double *out, int blocks, int iters, cudaStream_t st);
size_t step_smem_bytes(int MD, int nc, int kb);
bool pick_step_tiles(int MD, size_t budget, int *nc, int *kb);
size_t step_static_smem();
cudaError_t launch_schedule(const Params &P, int mode, cudaStream_t st);
cudaError_t launch_observe(const Params &P, int dump, int is_start, cudaStream_t st);
cudaError_t launch_init_state(const Params &P, cudaStream_t st, int tr0 = 0, int tr1 = -1);
cudaError_t launch_rk_schedule(const Params &P, cudaStream_t st);
cudaError_t launch_purity(const Params &P, double2 *hat, double2 *rho, double *out, cudaStream_t st);
cudaError_t launch_thresholds(const Params &P, cudaStream_t st, int tr0 = 0, int tr1 = -1);
cudaError_t launch_reset_times(const Params &P, cudaStream_t st);
cudaError_t launch_clear_records(const Params &P, cudaStream_t st);
cudaError_t launch_fp64_peak(double *out, int blocks, int iters, cudaStream_t st);
size_t split_smem_bytes(int MDs, int MD, int stages);
size_t split_stage_bytes(int MDs);
size_t split_static_smem();
cudaError_t launch_lpn(const Params &P, const LpnParams &L, int mode, double curr_time, int adr_dump,
                       cudaStream_t st);
}  // namespace qjx

// NVTX range around a host call (visible in Nsight Systems timelines; free when no tool is attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

using namespace qjx;

struct qjx_engine {
    qjx_config cfg{};
    Params P{};
    int MD = 0;
    int grid = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, eb0 = nullptr, eb1 = nullptr;
    std::string err;
    // device allocations
    std::vector<void *> allocs;
    size_t dev_bytes = 0;  // bytes of allocs
    double *d_inj_u = nullptr;
    long long *d_inj_off = nullptr;
    int *d_dump_at = nullptr;
    int dump_cap = 0;
    // ensemble purity scratch (allocated on the first qjx_purity call)
    double2 *d_hat = nullptr, *d_rho = nullptr;
    double *d_purity = nullptr;
    // host mirrors
    int *h_cnt = nullptr;   // pinned [G]
    int *h_ctrl = nullptr;  // pinned [16]: the control words [0, 8); split form: recheck counts [8, 11),
                            // micro-steps run [11], tiles of the next step [12]
    bool split_coop = true;  // split form: batches of micro-steps as one cooperative launch
    std::vector<std::vector<double>> jt, jn, je;
    std::vector<std::vector<int>> jtype;
    qjx_stats stats{};
    bool states_set = false;
    int period_base = 0;  // periods run since the last time reset (the RK propagator's period_id)
    int n_ens = 1;        // ensembles (qjx_create_batch)
    std::vector<double> branch_len;   // copy of qjx_config.branch_len
    std::vector<int> e_tr0;           // host copy of the ensembles' first trajectories [E + 1]
    std::vector<int> e_d_host;        // host copy of the ensembles' dimensions [E]
    unsigned char *d_bases = nullptr; // Lyapunov transient mask (bases of every ensemble)
    // serving engines (qjx_create_slots): every ensemble is a slot with room for d_cap and n_cap
    int slot_dcap = 0, slot_ncap = 0;
    std::vector<int> slot_n;          // trajectories of the loaded ensemble (0: free)
    unsigned char *d_active = nullptr;
    // Lyapunov task (allocated by the first qjx_lpn_start)
    LpnParams L{};
    bool lpn_alloc = false, lpn_started = false;
};

static void *dalloc(qjx_engine *h, size_t bytes)
{
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, bytes ? bytes : 16);
    h->allocs.push_back(p);
    h->dev_bytes += bytes ? bytes : 16;
    return p;
}

static qjx_status fail(qjx_engine *h, qjx_status s, const std::string &msg)
{
    if (h) h->err = msg;
    return s;
}

static qjx_status cuda_fail(qjx_engine *h, cudaError_t e, const char *where)
{
    return fail(h, QJX_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

extern "C" const char *qjx_status_string(qjx_status s)
{
    switch (s) {
    case QJX_OK: return "ok";
    case QJX_ERR_INVALID_ARG: return "invalid argument";
    case QJX_ERR_OOM: return "out of device memory";
    case QJX_ERR_NORM_GT_ONE: return "norm more than 1";
    case QJX_ERR_RNG_EXHAUSTED: return "injected uniform sequence exhausted";
    case QJX_ERR_ZERO_JUMP_WEIGHTS: return "all jump channels have zero weight";
    case QJX_ERR_TIMEOUT: return "bounded device wait gave up";
    case QJX_ERR_CUDA: return "CUDA error";
    case QJX_ERR_UNSUPPORTED: return "unsupported configuration";
    case QJX_ERR_STATE: return "call out of order";
    }
    return "unknown";
}

// The reason the calling thread's last engine creation failed (its handle no longer exists).
static thread_local std::string g_create_err;

extern "C" const char *qjx_last_error(const qjx_engine *h) { return h ? h->err.c_str() : g_create_err.c_str(); }

// Transposes row-major complex d x d matrices into the device layout mats[g][k][row]
// (rows padded to MD and k to an even count with zeros), so one K-slab is one contiguous
// TMA bulk copy and the last k pair of the FP64 MMA multiplies exact zeros.
static void pack_transposed(const double *M, int d, int MD, double *out)
{
    for (int i = 0; i < d; i++)
        for (int k = 0; k < d; k++) {
            out[2 * ((size_t)k * MD + i)] = M[2 * ((size_t)i * d + k)];
            out[2 * ((size_t)k * MD + i) + 1] = M[2 * ((size_t)i * d + k) + 1];
        }
}

// bf16 nearest (ties to even) of x with 8 significant bits; *val receives the rounded value.
static uint16_t bf16_round(double x, double *val)
{
    if (x == 0.0 || !std::isfinite(x)) {
        *val = 0.0;
        return 0;
    }
    const int e = std::ilogb(x);
    const double q = std::ldexp(std::nearbyint(std::ldexp(x, 7 - e)), e - 7);
    const float f = (float)q;  // exact: 8 significant bits
    uint32_t b;
    std::memcpy(&b, &f, 4);
    *val = q;
    return (uint16_t)(b >> 16);
}

// bf16 planes of a row-major complex d x d matrix in the order the split-precision kernel loads
// them: out[ks][plane][MDs rows x 16 k], planes Re hi, Re lo, Im hi, Im lo, k-step ks covering
// k = 16 ks .. 16 ks + 15; core matrices of 8 rows x 8 k (16 bytes a row), K-halves 64 elements
// apart and 8-row groups 128 elements apart (zero padded beyond d).
static void pack_split(const double *M, int d, int MDs, int KS, uint16_t *out)
{
    const size_t plane = (size_t)MDs * 16;
    for (int ks = 0; ks < KS; ks++)
        for (int r = 0; r < MDs; r++)
            for (int j = 0; j < 16; j++) {
                const int k = 16 * ks + j;
                double re = 0.0, im = 0.0;
                if (r < d && k < d) {
                    re = M[2 * ((size_t)r * d + k)];
                    im = M[2 * ((size_t)r * d + k) + 1];
                }
                double hv = 0.0, lv = 0.0;
                const size_t off = (size_t)(r & 7) * 8 + (size_t)(r >> 3) * 128 + (size_t)(j >> 3) * 64 + (j & 7);
                uint16_t *o = out + (size_t)ks * 4 * plane + off;
                o[0] = bf16_round(re, &hv);
                o[plane] = bf16_round(re - hv, &lv);
                o[2 * plane] = bf16_round(im, &hv);
                o[3 * plane] = bf16_round(im - hv, &lv);
            }
}

// Split-level steps of every branch of one ensemble: level 0 steps half of the branch head,
// every level halves it (qj_proc.cpp:15-24).  The head is T (a branch is half a period) or, for
// the deep tasks, the sub-period T / (2 deep_num_steps) (core.cpp:9934); with explicit branch
// durations it is 2 len_b / brep.
static void fill_dt(const qjx_config &c, double T, double *out)
{
    const int brep = c.deep_num_steps > 0 ? 2 * c.deep_num_steps : 1;
    for (int b = 0; b < c.num_branches; b++) {
        const double head = c.branch_len ? 2.0 * c.branch_len[b] / double(brep)
                                         : (c.deep_num_steps > 0 ? 0.5 * T / double(c.deep_num_steps) : T);
        double dt = head * 0.5;
        for (int l = 0; l < c.deep; l++) {
            dt *= 0.5;
            out[(size_t)b * c.deep + l] = dt;
        }
    }
}

// One ensemble of an engine: its dimension, trajectories, period, Philox key and first stream,
// and operators (U: [num_branches][deep][d][d], L: [num_diss][d][d], g: [num_diss], HE, R).
struct EnsDesc {
    int d, n;
    double T;
    uint64_t seed;
    int64_t sbase;
    const double *U, *L, *g, *HE, *R;
};

template <class T>
static T *upload(qjx_engine *h, const std::vector<T> &v)
{
    T *p = (T *)dalloc(h, std::max<size_t>(1, v.size()) * sizeof(T));
    if (p && !v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
}

// ---------------------------------------------------------------- tile shapes
// Whether the plain kernel can run sub-tiles of nc columns and slabs of kb k rows for padded rows
// MD within `budget` bytes of dynamic shared memory (the constraints pick_step_tiles applies).
static bool tiles_fit(int MD, size_t budget, int nc, int kb)
{
    if (nc != 8 && nc != 16 && nc != 32) return false;
    if (kb < 2 || kb > kKB || (kb & 1)) return false;
    const int RB = MD / 8, W1 = 16 / (nc / 8);
    if ((RB + W1 - 1) / W1 > 8) return false;
    return step_smem_bytes(MD, nc, kb) <= budget;
}

// The autotuner's cache: text lines "precision d nc kb stages rows us" (later lines win), in
// $QJX_TILE_CACHE or $HOME/.cache/qjx_b200/tiles.txt.
static std::string tile_cache_path()
{
    if (const char *p = getenv("QJX_TILE_CACHE")) return p;
    if (const char *home = getenv("HOME")) return std::string(home) + "/.cache/qjx_b200/tiles.txt";
    return std::string();
}

static bool tile_cache_get(int precision, int d, qjx_tiles *t)
{
    const std::string fn = tile_cache_path();
    if (fn.empty()) return false;
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) return false;
    bool found = false;
    char line[256];
    while (fgets(line, sizeof line, f)) {
        int pr = 0, dd = 0;
        qjx_tiles x{};
        double us = 0.0;
        if (sscanf(line, "%d %d %d %d %d %d %lf", &pr, &dd, &x.nc, &x.kb, &x.stages, &x.rows, &us) == 7 &&
            pr == precision && dd == d) {
            *t = x;
            found = true;
        }
    }
    fclose(f);
    return found;
}

static void tile_cache_put(int precision, int d, const qjx_tiles &t, double us)
{
    const std::string fn = tile_cache_path();
    if (fn.empty()) return;
    const size_t slash = fn.rfind('/');
    if (slash != std::string::npos && slash > 0) {  // create the directory chain
        const std::string dir = fn.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); i++)
            if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    FILE *f = fopen(fn.c_str(), "a");
    if (!f) return;
    fprintf(f, "%d %d %d %d %d %d %.6f\n", precision, d, t.nc, t.kb, t.stages, t.rows, us);
    fclose(f);
}

// Engine over E ensembles (E = 1: an ordinary engine).  cfg supplies what the ensembles share:
// deep, num_branches, num_diss, num_robs, record, rng_kind, rec_cap, keep_adr, max_dumps,
// device, precision, deep_num_steps.
static qjx_status create_engine(const qjx_config *cfg, const std::vector<EnsDesc> &ens, int psi_slots,
                                qjx_engine **out)
{
    if (!cfg || !out || ens.empty()) return QJX_ERR_INVALID_ARG;
    *out = nullptr;
    const qjx_config &c = *cfg;
    if (c.deep < 1 || c.deep > 62 || c.num_branches < 1 || c.num_diss < 1 || c.num_robs < 0 || c.deep_num_steps < 0)
        return QJX_ERR_INVALID_ARG;
    const int E = (int)ens.size();
    int dmax = 0;
    long long ntot = 0;
    for (const EnsDesc &e : ens) {
        if (e.d < 2 || e.n < 1 || !(e.T > 0.0) || !e.U || !e.L || !e.g || !e.HE || (c.num_robs > 0 && !e.R))
            return QJX_ERR_INVALID_ARG;
        dmax = std::max(dmax, e.d);
        ntot += e.n;
    }
    const int Ge = c.num_branches * c.deep + c.num_diss + 1 + c.num_robs;  // groups per ensemble
    const long long Gl = (long long)E * Ge;
    if (dmax > kMaxMD || Gl > (1 << 24) || ntot > (1 << 30)) return QJX_ERR_UNSUPPORTED;
    if (c.precision != 0 && c.precision != 1) return QJX_ERR_INVALID_ARG;
    // the split kernel's N = MDs <= 256 and its shared-memory bucket tables hold one ensemble of
    // at most kMaxGroups matrices
    if (c.precision == 1 && dmax > 256) return QJX_ERR_UNSUPPORTED;
    const int G = (int)Gl;
    const int n = (int)ntot;

    qjx_engine *h = new (std::nothrow) qjx_engine();
    if (!h) return QJX_ERR_OOM;
    h->cfg = c;
    if (c.branch_len) {  // keep a copy: the caller's array need not outlive the call
        for (int b = 0; b < c.num_branches; b++)
            if (!(c.branch_len[b] > 0.0)) {
                delete h;
                return QJX_ERR_INVALID_ARG;
            }
        h->branch_len.assign(c.branch_len, c.branch_len + c.num_branches);
        h->cfg.branch_len = h->branch_len.data();
    }
    h->cfg.d = dmax;
    h->cfg.n_traj = n;
    h->n_ens = E;
    if (h->cfg.rec_cap <= 0) h->cfg.rec_cap = 1024;
    if (h->cfg.max_dumps <= 0) h->cfg.max_dumps = 1;
    auto bail = [&](qjx_status s) {
        qjx_destroy(h);
        return s;
    };
    auto bail_cuda = [&](cudaError_t e, const char *where) {
        g_create_err = std::string(where) + ": " + cudaGetErrorString(e);
        return bail(QJX_ERR_CUDA);
    };
    g_create_err.clear();
    if (cudaError_t e = cudaSetDevice(c.device); e != cudaSuccess) return bail_cuda(e, "cudaSetDevice");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    h->grid = sms > 0 ? sms : 148;
    // QJX_SPLIT_COOP=0: run the split form's micro-steps as one launch each (the path taken when a
    // cooperative launch cannot make every CTA resident)
    if (const char *v = getenv("QJX_SPLIT_COOP")) h->split_coop = v[0] != '0';
    if (cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking); e != cudaSuccess)
        return bail_cuda(e, "cudaStreamCreateWithFlags");
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    cudaEventCreate(&h->eb0);
    cudaEventCreate(&h->eb1);

    const int d = dmax;
    int rows_per_block = 0;
    const int MD = pick_layout(d, &rows_per_block);
    h->MD = MD;
    Params &P = h->P;
    std::vector<int> e_nc(E), e_kb(E);
    {  // plain step kernel tiling of every ensemble within the shared memory
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device);
        const size_t fixed = step_static_smem() + 1024;
        if ((size_t)optin <= fixed) return bail(QJX_ERR_UNSUPPORTED);
        size_t smem = 0;
        const size_t budget = (size_t)optin - fixed;
        for (int e = 0; e < E; e++) {
            const int MDe = 8 * ((ens[e].d + 7) / 8);
            qjx_tiles ct{};
            if (c.tiles.nc > 0 || c.tiles.kb > 0) {  // explicit shapes must fit
                if (!tiles_fit(MDe, budget, c.tiles.nc, c.tiles.kb)) return bail(QJX_ERR_UNSUPPORTED);
                e_nc[e] = c.tiles.nc;
                e_kb[e] = c.tiles.kb;
            } else if (tile_cache_get(0, ens[e].d, &ct) && tiles_fit(MDe, budget, ct.nc, ct.kb)) {
                e_nc[e] = ct.nc;  // the autotuner's choice for this dimension
                e_kb[e] = ct.kb;
            } else if (!pick_step_tiles(MDe, budget, &e_nc[e], &e_kb[e])) {
                return bail(QJX_ERR_UNSUPPORTED);
            }
            smem = std::max(smem, step_smem_bytes(MDe, e_nc[e], e_kb[e]));
        }
        P.step_smem = (int)smem;
    }
    P.d = d;
    P.MD = MD;
    P.n = n;
    P.deep = c.deep;
    P.nb = c.num_branches;
    P.nd = c.num_diss;
    P.nr = c.num_robs;
    P.G = G;
    P.E = E;
    P.gL0 = c.num_branches * c.deep;  // local group offsets, the same in every ensemble
    P.gHE = P.gL0 + c.num_diss;
    P.gR0 = P.gHE + 1;
    P.rng_kind = c.rng_kind;
    P.seed = ens[0].seed;
    P.tr_base = ens[0].sbase;
    P.keep_adr = c.keep_adr;
    P.rec_cap = h->cfg.rec_cap;
    P.n_active = n;

    // ensemble tables; matrices of ensemble e in its own transposed padded layout
    // [k < kp_e][row < MD_e] (zero padded), one after another
    std::vector<int> e_d(E), e_tr0(E + 1), e_g0(E), g_ens(G);
    std::vector<double> e_dt((size_t)E * c.num_branches * c.deep), e_rate((size_t)E * c.num_diss);
    std::vector<unsigned long long> e_seed(E);
    std::vector<long long> e_sbase(E), g_off(G), g_loff(G);
    long long moff = 0, loff = 0;
    e_tr0[0] = 0;
    for (int e = 0; e < E; e++) {
        const EnsDesc &x = ens[e];
        e_d[e] = x.d;
        e_tr0[e + 1] = e_tr0[e] + x.n;
        e_g0[e] = e * Ge;
        e_seed[e] = x.seed;
        e_sbase[e] = x.sbase;
        fill_dt(h->cfg, x.T, e_dt.data() + (size_t)e * c.num_branches * c.deep);
        for (int i = 0; i < c.num_diss; i++) e_rate[(size_t)e * c.num_diss + i] = x.g[i];
        const long long per = (long long)((x.d + 1) & ~1) * (8 * ((x.d + 7) / 8));
        for (int l = 0; l < Ge; l++) {
            g_ens[e * Ge + l] = e;
            g_off[e * Ge + l] = moff;
            g_loff[e * Ge + l] = loff;
            moff += per;
            loff += x.n;
        }
    }
    std::vector<double> host((size_t)moff * 2, 0.0);
    for (int e = 0; e < E; e++) {
        const EnsDesc &x = ens[e];
        const int MDe = 8 * ((x.d + 7) / 8);
        const size_t dd2 = (size_t)x.d * x.d * 2;
        auto dst = [&](int l) { return host.data() + 2 * (size_t)g_off[e * Ge + l]; };
        for (int b = 0; b < c.num_branches; b++)
            for (int l = 0; l < c.deep; l++)
                pack_transposed(x.U + dd2 * ((size_t)b * c.deep + l), x.d, MDe, dst(b * c.deep + l));
        for (int i = 0; i < c.num_diss; i++) pack_transposed(x.L + dd2 * i, x.d, MDe, dst(P.gL0 + i));
        pack_transposed(x.HE, x.d, MDe, dst(P.gHE));
        for (int i = 0; i < c.num_robs; i++) pack_transposed(x.R + dd2 * i, x.d, MDe, dst(P.gR0 + i));
    }
    double2 *mats = (double2 *)dalloc(h, host.size() * sizeof(double));
    if (!mats) return bail(QJX_ERR_OOM);
    cudaMemcpy(mats, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice);
    P.mats = mats;
    h->e_tr0 = e_tr0;
    h->e_d_host = e_d;
    P.e_d = upload(h, e_d);
    P.e_nc = upload(h, e_nc);
    P.e_kb = upload(h, e_kb);
    P.e_tr0 = upload(h, e_tr0);
    P.e_g0 = upload(h, e_g0);
    P.e_dt = upload(h, e_dt);
    P.e_rate = upload(h, e_rate);
    P.e_seed = upload(h, e_seed);
    P.e_sbase = upload(h, e_sbase);
    P.g_off = upload(h, g_off);
    P.g_ens = upload(h, g_ens);
    P.g_loff = upload(h, g_loff);
    P.ltot = loff;
    P.dt = P.e_dt;
    P.g = P.e_rate;
    P.plan = (int *)dalloc(h, (size_t)(2 * G + 2) * sizeof(int));
    P.plan_sync = (unsigned int *)dalloc(h, sizeof(unsigned int));
    if (!P.e_d || !P.e_nc || !P.e_kb || !P.e_tr0 || !P.e_g0 || !P.e_dt || !P.e_rate || !P.e_seed || !P.e_sbase || !P.g_off || !P.g_ens ||
        !P.g_loff || !P.plan || !P.plan_sync)
        return bail(QJX_ERR_OOM);
    cudaMemset(P.plan, 0, (size_t)(2 * G + 2) * sizeof(int));
    cudaMemset(P.plan_sync, 0, sizeof(unsigned int));

    P.grid = h->grid;
    if (c.precision == 1) {  // split precision: bf16 planes of every matrix in the tcgen05 order
        P.split = 1;
        std::vector<int> e_mds(E), e_ks(E);
        int mds_max = 16;
        for (int e = 0; e < E; e++) {
            e_mds[e] = 16 * ((ens[e].d + 15) / 16);
            e_ks[e] = (ens[e].d + 15) / 16;
            mds_max = std::max(mds_max, e_mds[e]);
        }
        P.MDs = mds_max;
        P.KS = (d + 15) / 16;
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device);
        // deepest operand ring (2..8 stages) that fits next to the kernel's static shared memory
        const size_t fixed = split_static_smem() + 1024;
        int smax = 0;
        for (int st = kMaxSplitStages; st >= 2 && !smax; st--)
            if (split_smem_bytes(P.MDs, MD, st) + fixed <= (size_t)optin) smax = st;
        if (!smax) return bail(QJX_ERR_UNSUPPORTED);
        qjx_tiles ct{};
        const bool cached = !c.tiles.stages && !c.tiles.rows && tile_cache_get(1, d, &ct);
        const int want_st = c.tiles.stages ? c.tiles.stages : (cached ? ct.stages : smax);
        const int want_rows = c.tiles.rows ? c.tiles.rows : (cached ? ct.rows : 8);
        if (want_st < 2 || want_st > smax || want_rows < 8 || want_rows > 128 || (want_rows & 7))
            return bail(QJX_ERR_UNSUPPORTED);
        P.sstages = want_st;
        P.min_rows = want_rows;
        // per group: its bf16 matrix planes (usplit) in its ensemble's own padded layout
        std::vector<long long> uoff(G);
        size_t ubytes = 0;
        for (int gg = 0; gg < G; gg++) {
            const int e = g_ens[gg];
            uoff[gg] = (long long)ubytes;
            ubytes += (size_t)e_ks[e] * 4 * (size_t)e_mds[e] * 32;
        }
        P.e_mds = upload(h, e_mds);
        P.e_ks = upload(h, e_ks);
        P.g_uoff = upload(h, uoff);
        P.splan = (int *)dalloc(h, (size_t)(G + 2) * sizeof(int));
        // near-threshold FP64 rechecks: lists, band, and the matrix slab height that fits the ring
        // next to the input and product vectors
        P.rcnt = (int *)dalloc(h, 3 * sizeof(int));
        P.rlist = (int *)dalloc(h, (size_t)2 * n * sizeof(int));
        P.gen = (unsigned int *)dalloc(h, sizeof(unsigned int));
        P.sdone = (int *)dalloc(h, sizeof(int));
        if (!P.e_mds || !P.e_ks || !P.g_uoff || !P.splan || !P.rcnt || !P.rlist || !P.gen || !P.sdone)
            return bail(QJX_ERR_OOM);
        cudaMemset(P.gen, 0, sizeof(unsigned int));
        cudaMemset(P.sdone, 0, sizeof(int));
        P.recheck_tol = c.split_recheck == 0.0 ? 1e-5 : (c.split_recheck < 0.0 ? 0.0 : c.split_recheck);
        const size_t ring = (size_t)P.sstages * split_stage_bytes(P.MDs);
        const size_t vec = (size_t)(2 * MD + 2) * sizeof(double2);
        P.rchk_kb = std::min<int>(32, (int)((ring - vec) / (2 * (size_t)MD * sizeof(double2)))) & ~1;
        if (P.rchk_kb < 2) return bail(QJX_ERR_UNSUPPORTED);
        std::vector<uint16_t> hs(ubytes / 2, 0);
        for (int e = 0; e < E; e++) {
            const EnsDesc &x = ens[e];
            const size_t dd2 = (size_t)x.d * x.d * 2;
            auto dst = [&](int l) { return hs.data() + uoff[e * Ge + l] / 2; };
            for (int b = 0; b < c.num_branches; b++)
                for (int l = 0; l < c.deep; l++)
                    pack_split(x.U + dd2 * ((size_t)b * c.deep + l), x.d, e_mds[e], e_ks[e], dst(b * c.deep + l));
            for (int i = 0; i < c.num_diss; i++) pack_split(x.L + dd2 * i, x.d, e_mds[e], e_ks[e], dst(P.gL0 + i));
            pack_split(x.HE, x.d, e_mds[e], e_ks[e], dst(P.gHE));
            for (int i = 0; i < c.num_robs; i++) pack_split(x.R + dd2 * i, x.d, e_mds[e], e_ks[e], dst(P.gR0 + i));
        }
        unsigned char *us = (unsigned char *)dalloc(h, std::max<size_t>(ubytes, 16));
        if (!us) return bail(QJX_ERR_OOM);
        cudaMemcpy(us, hs.data(), ubytes, cudaMemcpyHostToDevice);
        P.usplit = us;
    }
    P.brep = c.deep_num_steps > 0 ? 2 * c.deep_num_steps : 1;

    P.psi = (double2 *)dalloc(h, (size_t)psi_slots * n * MD * sizeof(double2));
    P.st = (TrajState *)dalloc(h, (size_t)n * sizeof(TrajState));
    P.gn = (double *)dalloc(h, (size_t)n * c.num_diss * sizeof(double));
    P.cnt = (int *)dalloc(h, (size_t)3 * G * sizeof(int));
    P.lists = (int *)dalloc(h, (size_t)2 * P.ltot * sizeof(int));
    const size_t nd_ = (size_t)h->cfg.max_dumps * n;
    P.o_norm = (double *)dalloc(h, nd_ * sizeof(double));
    P.o_mean = (double *)dalloc(h, nd_ * sizeof(double));
    P.o_disp = (double *)dalloc(h, nd_ * sizeof(double));
    P.o_m2 = (double *)dalloc(h, nd_ * sizeof(double));
    P.o_energy = (double *)dalloc(h, nd_ * sizeof(double));
    P.o_robs = (double2 *)dalloc(h, nd_ * std::max(1, c.num_robs) * sizeof(double2));
    P.o_adr = (double *)dalloc(h, (c.keep_adr ? nd_ : (size_t)n) * d * sizeof(double));
    P.mean_start = (double *)dalloc(h, (size_t)n * sizeof(double));
    const size_t rc = (size_t)P.rec_cap * n;
    P.r_time = (double *)dalloc(h, rc * sizeof(double));
    P.r_norm = (double *)dalloc(h, rc * sizeof(double));
    P.r_eta = (double *)dalloc(h, rc * sizeof(double));
    P.r_type = (int *)dalloc(h, rc * sizeof(int));
    P.ctrl = (int *)dalloc(h, 16 * sizeof(int));
    P.work = (long long *)dalloc(h, 4 * sizeof(long long));
    if (!P.psi || !P.st || !P.gn || !P.cnt || !P.lists || !P.o_norm || !P.o_mean || !P.o_disp || !P.o_m2 ||
        !P.o_energy || !P.o_robs || !P.o_adr || !P.mean_start || !P.r_time || !P.r_norm || !P.r_eta || !P.r_type ||
        !P.ctrl || !P.work)
        return bail(QJX_ERR_OOM);
    if (cudaMallocHost(&h->h_cnt, sizeof(int) * G) != cudaSuccess ||
        cudaMallocHost(&h->h_ctrl, sizeof(int) * 16) != cudaSuccess)
        return bail(QJX_ERR_OOM);
    h->jt.assign(n, {});
    h->jn.assign(n, {});
    h->je.assign(n, {});
    h->jtype.assign(n, {});
    // the setup's memsets and copies ran on the legacy default stream; the engine's stream does not
    // wait for it (and a device-wide sync would wait for every other engine in the process)
    if (cudaError_t e = cudaStreamSynchronize(0); e != cudaSuccess) return bail_cuda(e, "engine setup");
    if (cudaError_t e = launch_init_state(P, h->stream); e != cudaSuccess) return bail_cuda(e, "init_state launch");
    if (cudaError_t e = cudaStreamSynchronize(h->stream); e != cudaSuccess) return bail_cuda(e, "init_state");
    *out = h;
    return QJX_OK;
}

// The ordinary engine: one ensemble described by cfg.
static qjx_status create_engine(const qjx_config *cfg, const double *U, const double *L, const double *g,
                                const double *HE, const double *R, int psi_slots, qjx_engine **out)
{
    if (!cfg || !out || !U || !L || !g || !HE) return QJX_ERR_INVALID_ARG;
    const qjx_config &c = *cfg;
    if (c.d < 2 || c.n_traj < 1 || !(c.T > 0.0) || (c.num_robs > 0 && !R)) return QJX_ERR_INVALID_ARG;
    if (c.d > kMaxMD) return QJX_ERR_UNSUPPORTED;
    const EnsDesc e{c.d, c.n_traj, c.T, c.seed, c.tr_base, U, L, g, HE, R};
    return create_engine(cfg, std::vector<EnsDesc>{e}, psi_slots, out);
}

extern "C" void qjx_destroy(qjx_engine *h)
{
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void *p : h->allocs) cudaFree(p);
    if (h->d_inj_u) cudaFree(h->d_inj_u);
    if (h->d_inj_off) cudaFree(h->d_inj_off);
    if (h->d_dump_at) cudaFree(h->d_dump_at);
    if (h->h_cnt) cudaFreeHost(h->h_cnt);
    if (h->h_ctrl) cudaFreeHost(h->h_ctrl);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->eb0) cudaEventDestroy(h->eb0);
    if (h->eb1) cudaEventDestroy(h->eb1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" qjx_status qjx_set_states(qjx_engine *h, const double *psi)
{
    if (!h || !psi) return QJX_ERR_INVALID_ARG;
    const Params &P = h->P;
    CK(cudaSetDevice(h->cfg.device));
    // every slot, so the rows past d that the gathers of odd d read are zero
    const int slots = P.prop == 1 ? kRkSlots : 2;
    CK(cudaMemsetAsync(P.psi, 0, (size_t)slots * P.n * P.MD * sizeof(double2), h->stream));
    CK(cudaMemcpy2DAsync(P.psi, (size_t)P.MD * sizeof(double2), psi, (size_t)P.d * sizeof(double2),
                         (size_t)P.d * sizeof(double2), P.n, cudaMemcpyHostToDevice, h->stream));
    CK(launch_init_state(P, h->stream));
    CK(cudaMemsetAsync(P.ctrl, 0, 16 * sizeof(int), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < P.n; i++) {
        h->jt[i].clear();
        h->jn[i].clear();
        h->je[i].clear();
        h->jtype[i].clear();
    }
    h->states_set = true;
    return QJX_OK;
}

extern "C" qjx_status qjx_set_uniforms(qjx_engine *h, const double *u, const int64_t *offsets)
{
    if (!h || !u || !offsets) return QJX_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->cfg.device));
    const int n = h->P.n;
    const int64_t total = offsets[n];
    if (offsets[0] != 0 || total < 0) return fail(h, QJX_ERR_INVALID_ARG, "offsets must start at 0");
    for (int i = 0; i < n; i++)
        if (offsets[i + 1] < offsets[i]) return fail(h, QJX_ERR_INVALID_ARG, "offsets must be non-decreasing");
    if (h->d_inj_u) cudaFree(h->d_inj_u);
    if (h->d_inj_off) cudaFree(h->d_inj_off);
    h->d_inj_u = nullptr;
    h->d_inj_off = nullptr;
    CK(cudaMalloc(&h->d_inj_u, std::max<int64_t>(total, 1) * sizeof(double)));
    CK(cudaMalloc(&h->d_inj_off, (size_t)(n + 1) * sizeof(long long)));
    CK(cudaMemcpy(h->d_inj_u, u, total * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_inj_off, offsets, (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice));
    h->P.inj_u = h->d_inj_u;
    h->P.inj_off = h->d_inj_off;
    return QJX_OK;
}

static qjx_status check_ctrl(qjx_engine *h)
{
    const int *c = h->h_ctrl;
    if (c[0] == 0) return QJX_OK;
    char buf[160];
    snprintf(buf, sizeof buf, "device error code %d on trajectory %d (%d errors)", c[3], c[1], c[0]);
    h->err = buf;
    switch (c[3]) {
    case ERR_NORM: return QJX_ERR_NORM_GT_ONE;
    case ERR_ZERO_W: return QJX_ERR_ZERO_JUMP_WEIGHTS;
    case ERR_RNG: return QJX_ERR_RNG_EXHAUSTED;
    case ERR_TIMEOUT: return QJX_ERR_TIMEOUT;
    default: return QJX_ERR_CUDA;
    }
}

extern "C" qjx_status qjx_init_thresholds(qjx_engine *h)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "qjx_set_states first");
    if (h->P.rng_kind == 1 && !h->P.inj_u) return fail(h, QJX_ERR_STATE, "qjx_set_uniforms first");
    CK(cudaSetDevice(h->cfg.device));
    CK(launch_thresholds(h->P, h->stream));
    CK(cudaMemcpyAsync(h->h_ctrl, h->P.ctrl, 16 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return check_ctrl(h);
}

extern "C" qjx_status qjx_reset_times(qjx_engine *h)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->cfg.device));
    CK(launch_reset_times(h->P, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->period_base = 0;
    return QJX_OK;
}

// Copies the device jump records into the per-trajectory host vectors and empties the
// device buffers.
static qjx_status drain_records(qjx_engine *h)
{
    const Params &P = h->P;
    if (!P.record) return QJX_OK;
    const int n = P.n;
    std::vector<TrajState> st(n);
    CK(cudaMemcpyAsync(st.data(), P.st, n * sizeof(TrajState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int maxrec = 0;
    for (int i = 0; i < n; i++) maxrec = std::max(maxrec, st[i].nrec);
    if (maxrec == 0) return QJX_OK;
    const size_t cntv = (size_t)maxrec * n;
    std::vector<double> t(cntv), nr(cntv), e(cntv);
    std::vector<int> ty(cntv);
    CK(cudaMemcpyAsync(t.data(), P.r_time, cntv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(nr.data(), P.r_norm, cntv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(e.data(), P.r_eta, cntv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(ty.data(), P.r_type, cntv * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < n; i++)
        for (int r = 0; r < st[i].nrec; r++) {
            const size_t o = (size_t)r * n + i;
            h->jt[i].push_back(t[o]);
            h->jn[i].push_back(nr[o]);
            h->je[i].push_back(e[o]);
            h->jtype[i].push_back(ty[o]);
        }
    CK(launch_clear_records(P, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->stats.jumps += (int64_t)0;
    return QJX_OK;
}

// Runs lock-step micro-steps until every trajectory is done for this call.  Step 0 of the
// call reads buckets written into cnt[0] / lists[0] by the schedule or observe kernel.
static qjx_status run_until_idle(qjx_engine *h)
{
    Params &P = h->P;
    // plain form: CUDA graphs of 6 micro-steps; split form: one cooperative launch runs up to
    // 6 x batch micro-steps with grid barriers between them (the buffers rotate with period 6)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (!P.split) {
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < 6; s++) {
            cudaError_t e = launch_step(P, s, h->grid, h->stream);
            if (e != cudaSuccess) {
                cudaStreamEndCapture(h->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                return cuda_fail(h, e, "launch_step");
            }
        }
        CK(cudaStreamEndCapture(h->stream, &graph));
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return cuda_fail(h, ie, "cudaGraphInstantiate");
    }
    int s0 = 0;  // split form: index of the next micro-step
    int64_t nlaunch = 0;

    qjx_status rs = QJX_OK;
    int batch = 1;
    // QJX_TRACE_BUCKETS=<file>: append the bucket sizes seen at every host poll (profiling aid)
    FILE *bucket_log = nullptr;
    if (const char *fn = getenv("QJX_TRACE_BUCKETS")) bucket_log = fopen(fn, "a");
    int64_t steps = 0;
    long long work0[3] = {0, 0, 0};
    cudaMemcpy(work0, P.work, 3 * sizeof(long long), cudaMemcpyDeviceToHost);
    cudaEventRecord(h->ev0, h->stream);
    while (true) {
        cudaEventRecord(h->eb0, h->stream);
        if (P.split) {
            cudaMemsetAsync(P.sdone, 0, sizeof(int), h->stream);
            cudaError_t e = h->split_coop ? launch_split_steps(P, s0, 6 * batch, h->grid, h->stream)
                                          : cudaErrorCooperativeLaunchTooLarge;
            if (e == cudaErrorCooperativeLaunchTooLarge) {
                // not every CTA can be resident (another context holds SMs): the same micro-steps
                // as one launch each (an empty step returns at once)
                cudaGetLastError();
                h->split_coop = false;
                e = cudaSuccess;
                for (int k = 0; k < 6 * batch && e == cudaSuccess; k++) e = launch_step(P, s0 + k, h->grid, h->stream);
                nlaunch += 6 * batch;
            } else {
                nlaunch += 1;
            }
            if (e != cudaSuccess) {
                rs = cuda_fail(h, e, "launch_split_steps");
                break;
            }
        } else {
            for (int b = 0; b < batch; b++) {
                cudaError_t e = cudaGraphLaunch(exec, h->stream);
                if (e != cudaSuccess) {
                    rs = cuda_fail(h, e, "cudaGraphLaunch");
                    break;
                }
            }
            if (rs != QJX_OK) break;
            steps += 6 * batch;
            nlaunch += 6 * batch;
        }
        cudaEventRecord(h->eb1, h->stream);
        // plain form: the next micro-step's plan total (or all bucket sizes for the bucket log),
        // which the last micro-step computed; split form: the micro-steps run, the recheck counts
        // and the next step's tiles
        const bool all_counts = !P.split && bucket_log;
        if (P.split) {
            cudaMemcpyAsync(h->h_ctrl + 8, P.rcnt, 3 * sizeof(int), cudaMemcpyDeviceToHost, h->stream);
            cudaMemcpyAsync(h->h_ctrl + 11, P.sdone, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
            cudaMemcpyAsync(h->h_ctrl + 12, P.splan + 1 + P.G, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        } else if (all_counts) {
            cudaMemcpyAsync(h->h_cnt, P.cnt, sizeof(int) * P.G, cudaMemcpyDeviceToHost, h->stream);
        } else {
            cudaMemcpyAsync(h->h_cnt, P.plan + P.G, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        }
        cudaMemcpyAsync(h->h_ctrl, P.ctrl, sizeof(int) * 8, cudaMemcpyDeviceToHost, h->stream);
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            rs = cuda_fail(h, e, "micro-step batch");
            break;
        }
        if (P.split) {
            steps += h->h_ctrl[11];
            s0 = (s0 + h->h_ctrl[11]) % 6;
        }
        float bms = 0.f;
        cudaEventElapsedTime(&bms, h->eb0, h->eb1);
        h->stats.step_kernel_ms += bms;
        rs = check_ctrl(h);
        if (rs != QJX_OK) break;
        long long active = all_counts ? 0 : h->h_cnt[0];
        if (all_counts)
            for (int g = 0; g < P.G; g++) active += h->h_cnt[g];
        // split form: tiles of the next step and trajectories waiting for an FP64 recheck
        if (P.split) active = (long long)h->h_ctrl[12] + h->h_ctrl[8 + s0 % 3];
        if (bucket_log && all_counts) {
            for (int g = 0; g < P.G; g++) fprintf(bucket_log, g ? " %d" : "%d", h->h_cnt[g]);
            fprintf(bucket_log, "\n");
        }
        if (active == 0) {
            if (h->h_ctrl[2] > 0) {  // paused on full record buffers: drain and resume
                rs = drain_records(h);
                if (rs != QJX_OK) break;
                cudaMemsetAsync(P.ctrl + 2, 0, sizeof(int), h->stream);
                cudaMemsetAsync(P.cnt, 0, sizeof(int) * 3 * P.G, h->stream);
                if (P.rcnt) cudaMemsetAsync(P.rcnt, 0, 3 * sizeof(int), h->stream);
                cudaError_t le = launch_schedule(P, 1, h->stream);
                h->stats.launches += 2;
                if (le != cudaSuccess) {
                    rs = cuda_fail(h, le, "launch_schedule");
                    break;
                }
                s0 = 0;  // the schedule wrote step 0's buckets
                continue;
            }
            break;
        }
        batch = std::min(batch * 2, 16);
    }
    if (bucket_log) fclose(bucket_log);
    cudaEventRecord(h->ev1, h->stream);
    cudaEventSynchronize(h->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.kernel_ms += ms;
    h->stats.last_call_ms = ms;
    h->stats.micro_steps += steps;
    h->stats.launches += nlaunch;
    long long work1[3] = {0, 0, 0};
    cudaMemcpy(work1, P.work, 3 * sizeof(long long), cudaMemcpyDeviceToHost);
    h->stats.matvecs += work1[0] - work0[0];
    h->stats.mma_tiles += work1[1] - work0[1];
    h->stats.rechecks += work1[2] - work0[2];
    if (exec) cudaGraphExecDestroy(exec);
    return rs;
}

extern "C" qjx_status qjx_create(const qjx_config *cfg, const double *U, const double *L, const double *g,
                                 const double *HE, const double *R, qjx_engine **out)
{
    return create_engine(cfg, U, L, g, HE, R, 2, out);
}

extern "C" qjx_status qjx_create_batch(const qjx_config *cfg, int n_ens, const qjx_ensemble *ens, qjx_engine **out)
{
    if (!cfg || !out || n_ens < 1 || !ens) return QJX_ERR_INVALID_ARG;
    std::vector<EnsDesc> v(n_ens);
    for (int e = 0; e < n_ens; e++) {
        const qjx_ensemble &x = ens[e];
        if (x.d > kMaxMD) return QJX_ERR_UNSUPPORTED;
        v[e] = EnsDesc{x.d, x.n_traj, x.T, x.seed, x.tr_base, x.U, x.L, x.g, x.HE, x.R};
    }
    return create_engine(cfg, v, 2, out);
}

extern "C" qjx_status qjx_create_slots(const qjx_config *cfg, int n_slots, int d_cap, int n_cap, qjx_engine **out)
{
    if (!cfg || !out || n_slots < 1 || d_cap < 2 || n_cap < 1) return QJX_ERR_INVALID_ARG;
    if (cfg->precision != 0 || d_cap > kMaxMD) return QJX_ERR_UNSUPPORTED;
    const qjx_config &c = *cfg;
    // placeholder operators (zero) until a slot is loaded
    const size_t dd2 = (size_t)2 * d_cap * d_cap;
    std::vector<double> U(dd2 * c.num_branches * std::max(1, c.deep)), L(dd2 * std::max(1, c.num_diss)), HE(dd2),
        R(dd2 * std::max(1, c.num_robs)), g(std::max(1, c.num_diss), 1.0);
    std::vector<EnsDesc> v(n_slots, EnsDesc{d_cap, n_cap, 1.0, 0, 0, U.data(), L.data(), g.data(), HE.data(),
                                            c.num_robs ? R.data() : nullptr});
    qjx_status st = create_engine(cfg, v, 2, out);
    if (st != QJX_OK) return st;
    qjx_engine *h = *out;
    h->slot_dcap = d_cap;
    h->slot_ncap = n_cap;
    h->slot_n.assign(n_slots, 0);
    h->d_active = (unsigned char *)dalloc(h, (size_t)h->P.n);
    if (!h->d_active) {
        qjx_destroy(h);
        *out = nullptr;
        return QJX_ERR_OOM;
    }
    cudaMemset(h->d_active, 0, (size_t)h->P.n);
    h->P.active = h->d_active;
    h->states_set = true;
    return QJX_OK;
}

extern "C" qjx_status qjx_slot_load(qjx_engine *h, int slot, const qjx_ensemble *e, const double *psi)
{
    NvtxRange range("qjx_slot_load");
    if (!h || !e) return QJX_ERR_INVALID_ARG;
    if (!h->d_active || slot < 0 || slot >= h->n_ens) return fail(h, QJX_ERR_INVALID_ARG, "not a slot of a serving engine");
    if (h->slot_n[slot]) return fail(h, QJX_ERR_STATE, "slot in use: release it first");
    Params &P = h->P;
    const int d = e->d, n = e->n_traj;
    if (d < 2 || d > h->slot_dcap || n < 1 || n > h->slot_ncap || !(e->T > 0.0) || !e->U || !e->L || !e->g || !e->HE ||
        (P.nr > 0 && !e->R))
        return fail(h, QJX_ERR_INVALID_ARG, "ensemble does not fit the slot");
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaStreamSynchronize(h->stream));
    const int MDe = 8 * ((d + 7) / 8), kpe = (d + 1) & ~1;
    int nc = 0, kb = 0;
    qjx_tiles ct{};
    if (tile_cache_get(0, d, &ct) && tiles_fit(MDe, (size_t)P.step_smem, ct.nc, ct.kb)) {
        nc = ct.nc;  // the autotuner's choice for this dimension
        kb = ct.kb;
    } else if (!pick_step_tiles(MDe, (size_t)P.step_smem, &nc, &kb)) {
        return fail(h, QJX_ERR_UNSUPPORTED, "no tiling");
    }
    // operators into the slot's resident matrix region
    const int Ge = P.G / h->n_ens;
    const size_t per = (size_t)kpe * MDe * 2, dd2 = (size_t)2 * d * d;
    std::vector<double> host(per * Ge, 0.0);
    for (int b = 0; b < P.nb; b++)
        for (int l = 0; l < P.deep; l++)
            pack_transposed(e->U + dd2 * ((size_t)b * P.deep + l), d, MDe, host.data() + per * (b * P.deep + l));
    for (int i = 0; i < P.nd; i++) pack_transposed(e->L + dd2 * i, d, MDe, host.data() + per * (P.gL0 + i));
    pack_transposed(e->HE, d, MDe, host.data() + per * P.gHE);
    for (int i = 0; i < P.nr; i++) pack_transposed(e->R + dd2 * i, d, MDe, host.data() + per * (P.gR0 + i));
    std::vector<long long> goff(Ge);
    CK(cudaMemcpy(goff.data(), P.g_off + (size_t)slot * Ge, Ge * sizeof(long long), cudaMemcpyDeviceToHost));
    for (int l = 0; l < Ge; l++)
        CK(cudaMemcpy(const_cast<double2 *>(P.mats) + goff[l], host.data() + per * l, per * sizeof(double),
                      cudaMemcpyHostToDevice));
    // the slot's ensemble table entries
    std::vector<double> dts((size_t)P.nb * P.deep);
    fill_dt(h->cfg, e->T, dts.data());
    const unsigned long long seed = e->seed;
    const long long sbase = e->tr_base;
    CK(cudaMemcpy(const_cast<int *>(P.e_d) + slot, &d, sizeof(int), cudaMemcpyHostToDevice));
    h->e_d_host[slot] = d;
    CK(cudaMemcpy(const_cast<int *>(P.e_nc) + slot, &nc, sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(const_cast<int *>(P.e_kb) + slot, &kb, sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(const_cast<double *>(P.e_dt) + (size_t)slot * P.nb * P.deep, dts.data(),
                  dts.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(const_cast<double *>(P.e_rate) + (size_t)slot * P.nd, e->g, P.nd * sizeof(double),
                  cudaMemcpyHostToDevice));
    CK(cudaMemcpy(const_cast<unsigned long long *>(P.e_seed) + slot, &seed, sizeof(seed), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(const_cast<long long *>(P.e_sbase) + slot, &sbase, sizeof(sbase), cudaMemcpyHostToDevice));
    // states: psi (or |0>) in rows of the largest dimension, fresh records, thresholds
    const int t0 = slot * h->slot_ncap;
    CK(cudaMemset(P.psi + (size_t)t0 * P.MD, 0, (size_t)h->slot_ncap * P.MD * sizeof(double2)));
    CK(cudaMemset(P.psi + ((size_t)P.n + t0) * P.MD, 0, (size_t)h->slot_ncap * P.MD * sizeof(double2)));
    if (psi) {
        CK(cudaMemcpy2D(P.psi + (size_t)t0 * P.MD, (size_t)P.MD * sizeof(double2), psi, (size_t)d * sizeof(double2),
                        (size_t)d * sizeof(double2), n, cudaMemcpyHostToDevice));
    } else {
        const double2 one = make_double2(1.0, 0.0);
        for (int i = 0; i < n; i++) CK(cudaMemcpy(P.psi + ((size_t)t0 + i) * P.MD, &one, sizeof(one), cudaMemcpyHostToDevice));
    }
    CK(launch_init_state(P, h->stream, t0, t0 + h->slot_ncap));
    CK(launch_thresholds(P, h->stream, t0, t0 + n));
    CK(cudaMemsetAsync(h->d_active + t0, 1, (size_t)n, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int i = t0; i < t0 + h->slot_ncap; i++) {
        h->jt[i].clear();
        h->jn[i].clear();
        h->je[i].clear();
        h->jtype[i].clear();
    }
    h->slot_n[slot] = n;
    return QJX_OK;
}

extern "C" qjx_status qjx_slot_release(qjx_engine *h, int slot)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    if (!h->d_active || slot < 0 || slot >= h->n_ens) return fail(h, QJX_ERR_INVALID_ARG, "not a slot of a serving engine");
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaMemset(h->d_active + (size_t)slot * h->slot_ncap, 0, (size_t)h->slot_ncap));
    h->slot_n[slot] = 0;
    return QJX_OK;
}

extern "C" qjx_status qjx_create_rk(const qjx_config *cfg, const double *H_eff, const double *H_drv, double E0,
                                    double A, int drv_type, double drv_freq, double drv_phase, int rk_ns,
                                    const double *L, const double *g, const double *HE, const double *R,
                                    qjx_engine **out)
{
    if (!cfg || !out || !H_eff || !H_drv || rk_ns < 1) return QJX_ERR_INVALID_ARG;
    if (cfg->precision != 0) return QJX_ERR_UNSUPPORTED;  // the RK propagator runs the FP64 plain form
    qjx_config c = *cfg;
    c.num_branches = 1;  // groups 0 and 1: H_eff and H_drv
    c.deep = 2;
    c.deep_num_steps = 0;
    c.branch_len = nullptr;
    const size_t dd2 = (size_t)2 * c.d * c.d;
    std::vector<double> M(2 * dd2);
    std::memcpy(M.data(), H_eff, dd2 * sizeof(double));
    std::memcpy(M.data() + dd2, H_drv, dd2 * sizeof(double));
    qjx_status st = create_engine(&c, M.data(), L, g, HE, R, kRkSlots, out);
    if (st != QJX_OK) return st;
    Params &P = (*out)->P;
    P.prop = 1;
    P.rk_ns = rk_ns;
    P.T = c.T;
    P.rk_step = c.T / double(rk_ns);  // init_rk (rk_proc.cpp:62)
    P.E0 = E0;
    P.A = A;
    P.drv_type = drv_type;
    P.drv_freq = drv_freq;
    P.drv_phase = drv_phase;
    return QJX_OK;
}

extern "C" qjx_status qjx_run_periods(qjx_engine *h, int n_periods, int is_obs, const int *dump_at, int n_dumps,
                                      int dump_base)
{
    NvtxRange range("qjx_run_periods");
    if (!h || n_periods < 0 || n_dumps < 0 || (n_dumps > 0 && !dump_at)) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "qjx_set_states first");
    if (dump_base < 0 || dump_base + n_dumps > h->cfg.max_dumps)
        return fail(h, QJX_ERR_INVALID_ARG, "dump slots exceed max_dumps");
    const int subdump = (h->cfg.deep_num_steps > 0 && is_obs == 1) ? 1 : 0;
    if (subdump && (n_dumps > 0 ||
                    dump_base + (long long)n_periods * h->cfg.num_branches * h->cfg.deep_num_steps > h->cfg.max_dumps))
        return fail(h, QJX_ERR_INVALID_ARG, "deep task: dump_at must be empty and every sub-period needs a dump slot");
    for (int i = 0; i < n_dumps; i++)
        if (dump_at[i] < 1 || dump_at[i] > n_periods || (i > 0 && dump_at[i] <= dump_at[i - 1]))
            return fail(h, QJX_ERR_INVALID_ARG, "dump_at must be ascending within 1..n_periods");
    if (n_periods == 0) return QJX_OK;
    CK(cudaSetDevice(h->cfg.device));
    Params &P = h->P;
    if (n_dumps > h->dump_cap) {
        if (h->d_dump_at) cudaFree(h->d_dump_at);
        h->d_dump_at = nullptr;
        CK(cudaMalloc(&h->d_dump_at, sizeof(int) * n_dumps));
        h->dump_cap = n_dumps;
    }
    if (n_dumps) CK(cudaMemcpy(h->d_dump_at, dump_at, sizeof(int) * n_dumps, cudaMemcpyHostToDevice));
    P.dump_at = h->d_dump_at;
    P.n_dumps = n_dumps;
    P.dump_base = dump_base;
    P.target = n_periods;
    P.subdump = subdump;
    P.record = (is_obs == 1 && h->cfg.record > 0) ? 1 : 0;
    CK(cudaMemsetAsync(P.cnt, 0, sizeof(int) * 3 * P.G, h->stream));
    if (P.rcnt) CK(cudaMemsetAsync(P.rcnt, 0, 3 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(P.ctrl, 0, sizeof(int) * 16, h->stream));
    P.period0 = h->period_base;
    if (P.prop == 1) CK(launch_rk_schedule(P, h->stream));
    else CK(launch_schedule(P, 0, h->stream));
    h->stats.launches += 1;
    qjx_status s = run_until_idle(h);
    if (s != QJX_OK) return s;
    h->period_base += n_periods;
    return drain_records(h);
}

// Deep tasks: continue every trajectory for n_sub sub-periods from where it stands, with the
// observables after each sub-period in dump slots dump_base, dump_base + 1, ... (the per-sub-period
// loop of ex_period_obs_deep_mult_lpn, core.cpp:155-241, which runs the Lyapunov update between
// sub-periods).  Periods continue across calls; a later qjx_run_periods starts a new period.
extern "C" qjx_status qjx_run_sub_periods(qjx_engine *h, int n_sub, int dump_base)
{
    NvtxRange range("qjx_run_sub_periods");
    if (!h || n_sub < 1 || dump_base < 0) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "qjx_set_states first");
    if (h->cfg.deep_num_steps < 1 || h->P.prop != 0)
        return fail(h, QJX_ERR_INVALID_ARG, "sub-periods exist for the deep tasks with the QJ propagator only");
    if ((long long)dump_base + n_sub > h->cfg.max_dumps)
        return fail(h, QJX_ERR_INVALID_ARG, "every sub-period needs a dump slot below max_dumps");
    CK(cudaSetDevice(h->cfg.device));
    Params &P = h->P;
    P.dump_at = h->d_dump_at;
    P.n_dumps = 0;
    P.dump_base = dump_base;
    P.target = 0x7fffffff;  // periods do not end the call; sub_target does
    P.sub_target = n_sub;
    P.subdump = 1;
    P.record = h->cfg.record > 0 ? 1 : 0;
    CK(cudaMemsetAsync(P.cnt, 0, sizeof(int) * 3 * P.G, h->stream));
    if (P.rcnt) CK(cudaMemsetAsync(P.rcnt, 0, 3 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(P.ctrl, 0, sizeof(int) * 16, h->stream));
    P.period0 = h->period_base;
    cudaError_t e = launch_schedule(P, 2, h->stream);
    h->stats.launches += 1;
    qjx_status st = e == cudaSuccess ? run_until_idle(h) : cuda_fail(h, e, "launch_schedule");
    P.sub_target = 0;
    if (st != QJX_OK) return st;
    return drain_records(h);
}

extern "C" qjx_status qjx_observe(qjx_engine *h, int dump, int is_start)
{
    NvtxRange range("qjx_observe");
    if (!h || dump < 0 || dump >= h->cfg.max_dumps) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "qjx_set_states first");
    CK(cudaSetDevice(h->cfg.device));
    Params &P = h->P;
    P.target = 0;
    P.n_dumps = 1;
    P.dump_base = dump;
    P.record = 0;
    P.subdump = 0;
    CK(cudaMemsetAsync(P.cnt, 0, sizeof(int) * 3 * P.G, h->stream));
    if (P.rcnt) CK(cudaMemsetAsync(P.rcnt, 0, 3 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(P.ctrl, 0, sizeof(int) * 16, h->stream));
    CK(launch_observe(P, dump, is_start, h->stream));
    h->stats.launches += 1;
    return run_until_idle(h);
}

extern "C" qjx_status qjx_get_observables(qjx_engine *h, int dump0, int n_dumps, double *norm, double *mean,
                                          double *dispersion, double *m2, double *energy, double *robs,
                                          double *adr)
{
    if (!h || dump0 < 0 || n_dumps < 0 || dump0 + n_dumps > h->cfg.max_dumps) return QJX_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->cfg.device));
    const Params &P = h->P;
    const size_t o = (size_t)dump0 * P.n, cnt = (size_t)n_dumps * P.n;
    if (norm) CK(cudaMemcpy(norm, P.o_norm + o, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    if (mean) CK(cudaMemcpy(mean, P.o_mean + o, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    if (dispersion) CK(cudaMemcpy(dispersion, P.o_disp + o, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    if (m2) CK(cudaMemcpy(m2, P.o_m2 + o, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    if (energy) CK(cudaMemcpy(energy, P.o_energy + o, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    if (robs && P.nr > 0)
        CK(cudaMemcpy(robs, P.o_robs + o * P.nr, cnt * P.nr * sizeof(double2), cudaMemcpyDeviceToHost));
    if (adr) {
        if (P.keep_adr)
            CK(cudaMemcpy(adr, P.o_adr + o * P.d, cnt * P.d * sizeof(double), cudaMemcpyDeviceToHost));
        else
            CK(cudaMemcpy(adr, P.o_adr, (size_t)P.n * P.d * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return QJX_OK;
}

extern "C" qjx_status qjx_purity(qjx_engine *h, double *purity, double *rho)
{
    if (!h || !purity) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "qjx_set_states first");
    if (h->n_ens != 1) return fail(h, QJX_ERR_UNSUPPORTED, "qjx_purity takes a single-ensemble engine");
    CK(cudaSetDevice(h->cfg.device));
    Params &P = h->P;
    if (!h->d_hat) {
        h->d_hat = (double2 *)dalloc(h, (size_t)P.n * P.MD * sizeof(double2));
        h->d_rho = (double2 *)dalloc(h, (size_t)P.d * P.d * sizeof(double2));
        h->d_purity = (double *)dalloc(h, sizeof(double));
        if (!h->d_hat || !h->d_rho || !h->d_purity) {
            h->d_hat = nullptr;
            return fail(h, QJX_ERR_OOM, "purity scratch");
        }
    }
    CK(launch_purity(P, h->d_hat, h->d_rho, h->d_purity, h->stream));
    h->stats.launches += 3;
    CK(cudaMemcpyAsync(purity, h->d_purity, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (rho)
        CK(cudaMemcpyAsync(rho, h->d_rho, (size_t)P.d * P.d * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return QJX_OK;
}

extern "C" qjx_status qjx_get_mean_start(qjx_engine *h, double *mean_start)
{
    if (!h || !mean_start) return QJX_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaMemcpy(mean_start, h->P.mean_start, h->P.n * sizeof(double), cudaMemcpyDeviceToHost));
    return QJX_OK;
}

extern "C" qjx_status qjx_get_states(qjx_engine *h, double *psi, double *t, double *eta, int *jumps_counts)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->cfg.device));
    const Params &P = h->P;
    std::vector<TrajState> st(P.n);
    CK(cudaMemcpy(st.data(), P.st, P.n * sizeof(TrajState), cudaMemcpyDeviceToHost));
    if (psi) {
        std::vector<double2> all((size_t)2 * P.n * P.MD);
        CK(cudaMemcpy(all.data(), P.psi, all.size() * sizeof(double2), cudaMemcpyDeviceToHost));
        for (int i = 0; i < P.n; i++)
            memcpy(psi + (size_t)2 * i * P.d, all.data() + ((size_t)st[i].cur * P.n + i) * P.MD,
                   (size_t)P.d * sizeof(double2));
    }
    for (int i = 0; i < P.n; i++) {
        if (t) t[i] = st[i].t;
        if (eta) eta[i] = st[i].eta;
        if (jumps_counts) jumps_counts[i] = st[i].jumps;
    }
    return QJX_OK;
}

extern "C" qjx_status qjx_jump_count(qjx_engine *h, int tr, int64_t *count)
{
    if (!h || !count || tr < 0 || tr >= h->P.n) return QJX_ERR_INVALID_ARG;
    *count = (int64_t)h->jt[tr].size();
    return QJX_OK;
}

extern "C" qjx_status qjx_get_jumps(qjx_engine *h, int tr, double *times, int *types, double *norms, double *etas)
{
    if (!h || tr < 0 || tr >= h->P.n) return QJX_ERR_INVALID_ARG;
    const size_t k = h->jt[tr].size();
    if (times) memcpy(times, h->jt[tr].data(), k * sizeof(double));
    if (types) memcpy(types, h->jtype[tr].data(), k * sizeof(int));
    if (norms) memcpy(norms, h->jn[tr].data(), k * sizeof(double));
    if (etas) memcpy(etas, h->je[tr].data(), k * sizeof(double));
    return QJX_OK;
}

extern "C" qjx_status qjx_get_stats(qjx_engine *h, qjx_stats *stats)
{
    if (!h || !stats) return QJX_ERR_INVALID_ARG;
    int64_t jumps = 0;
    for (auto &v : h->jt) jumps += (int64_t)v.size();
    h->stats.jumps = jumps;
    *stats = h->stats;
    return QJX_OK;
}

extern "C" qjx_status qjx_set_active(qjx_engine *h, int n_active)
{
    if (!h || n_active < 0 || n_active > h->P.n) return QJX_ERR_INVALID_ARG;
    h->P.n_active = n_active;
    return QJX_OK;
}

extern "C" qjx_status qjx_set_bases_only(qjx_engine *h, int on)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    if (h->d_active) return fail(h, QJX_ERR_UNSUPPORTED, "serving engines keep their slot mask");
    CK(cudaSetDevice(h->cfg.device));
    if (!on) {
        h->P.active = nullptr;
        return QJX_OK;
    }
    if (!h->d_bases) {
        std::vector<unsigned char> m(h->P.n, 0);
        for (int e = 0; e < h->n_ens; e++) {
            const int t0 = h->e_tr0[e], half = (h->e_tr0[e + 1] - t0) / 2;
            for (int i = 0; i < half; i++) m[t0 + i] = 1;
        }
        h->d_bases = upload(h, m);
        if (!h->d_bases) return fail(h, QJX_ERR_OOM, "bases mask");
    }
    h->P.active = h->d_bases;
    return QJX_OK;
}

extern "C" qjx_status qjx_lpn_start(qjx_engine *h, const qjx_lpn_config *c)
{
    if (!h || !c) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "qjx_set_states first");
    const Params &P = h->P;
    if (h->d_active) return fail(h, QJX_ERR_UNSUPPORTED, "the Lyapunov task does not run on serving slots");
    for (int e = 0; e < h->n_ens; e++) {
        const int ne = h->e_tr0[e + 1] - h->e_tr0[e];
        if (ne < 2 || (ne & 1))
            return fail(h, QJX_ERR_INVALID_ARG, "the Lyapunov task needs an even n_traj >= 2 in every ensemble");
    }
    const int cs = c->chars_sys;
    if (cs != 0 && cs != 1 && cs != 3 && cs != 5)
        return fail(h, QJX_ERR_INVALID_ARG, "chars_sys must be 0 (dimer), 1 (JCS), 3 (MBL) or 5 (Integrable)");
    if ((cs == 3) != (c->mbl_Nc != 0)) return fail(h, QJX_ERR_INVALID_ARG, "mbl_Nc goes with chars_sys 3 only");
    if (cs != 0 && (P.nr < 1 || !(c->spec_div != 0.0)))
        return fail(h, QJX_ERR_INVALID_ARG, "the spec operator goes in observable slot 0, with spec_div != 0");
    if (cs == 5 && c->lpn_type == -2) return fail(h, QJX_ERR_INVALID_ARG, "Integrable has no lpn_type -2");
    const int shift = cs != 0 ? 1 : 0;  // JCS / MBL / Integrable: slot 0 holds the spec operator
    if (!(c->lpn_type == -1 || c->lpn_type == -2 || (c->lpn_type >= 0 && c->lpn_type + shift < P.nr)))
        return fail(h, QJX_ERR_INVALID_ARG, "lpn_type must be -1, -2 or a random observable index");
    std::vector<int> words;
    if (c->mbl_Nc != 0) {
        int dm = 0;
        if (qjx_mbl_size(c->mbl_Nc, 0, &dm, nullptr) != QJX_OK || P.nr < 1 || !(c->spec_div != 0.0))
            return fail(h, QJX_ERR_INVALID_ARG, "mbl_Nc must be even in [2, 24] with H in observable slot 0");
        for (int e = 0; e < h->n_ens; e++)
            if (h->e_d_host[e] != dm) return fail(h, QJX_ERR_INVALID_ARG, "mbl_Nc does not match the dimension");
        for (int x = 0; x < (1 << c->mbl_Nc); x++)
            if (__builtin_popcount(x) == c->mbl_Nc / 2) words.push_back(x);
    }
    if (P.nr > 64) return fail(h, QJX_ERR_UNSUPPORTED, "the Lyapunov task takes at most 64 random observables");
    if (c->eps_deep < 0) return fail(h, QJX_ERR_INVALID_ARG, "eps_deep must be >= 0");
    CK(cudaSetDevice(h->cfg.device));
    LpnParams &L = h->L;
    const size_t n = P.n;
    if (!h->lpn_alloc) {
        L.lambda = (double *)dalloc(h, n * sizeof(double));
        L.lambda_now = (double *)dalloc(h, n * sizeof(double));
        L.delta_s_v = (double *)dalloc(h, n * sizeof(double));
        L.mean_lpn = (double *)dalloc(h, n * sizeof(double));
        L.energy_lpn = (double *)dalloc(h, n * sizeof(double));
        L.robs_lpn = (double2 *)dalloc(h, n * std::max(1, P.nr) * sizeof(double2));
        L.num_renorms = (int *)dalloc(h, n * sizeof(int));
        L.var_pos = (long long *)dalloc(h, n * sizeof(long long));
        L.renormed = (int *)dalloc(h, n * sizeof(int));
        L.ratio = (double *)dalloc(h, n * sizeof(double));
        L.ds_rec = (double *)dalloc(h, n * sizeof(double));
        L.df_rec = (double *)dalloc(h, n * sizeof(double));
        L.eps_iters = (int *)dalloc(h, n * sizeof(int));
        L.eps = (double *)dalloc(h, n * sizeof(double));
        std::vector<int> pair0(h->n_ens + 1, 0);
        for (int e = 0; e < h->n_ens; e++) pair0[e + 1] = pair0[e] + (h->e_tr0[e + 1] - h->e_tr0[e]) / 2;
        L.pair0 = upload(h, pair0);
        L.pairs = pair0[h->n_ens];
        if (!L.lambda || !L.lambda_now || !L.delta_s_v || !L.mean_lpn || !L.energy_lpn || !L.robs_lpn ||
            !L.num_renorms || !L.var_pos || !L.renormed || !L.ratio || !L.ds_rec || !L.df_rec || !L.eps_iters || !L.eps ||
            !L.pair0)
            return fail(h, QJX_ERR_OOM, "Lyapunov arrays");
        h->lpn_alloc = true;
    }
    L.lpn_type = c->lpn_type;
    L.eps_deep = c->eps_deep;
    L.per_period = c->per_period ? 1 : 0;
    L.eps_low = c->eps_low;
    L.eps_high = c->eps_high;
    L.eps_error = c->eps_error;
    L.delta_s = c->delta_s;
    L.delta_f_high = c->delta_f_high;
    L.delta_f_low = c->delta_f_low;
    L.max_energy = c->max_energy;
    L.mbl_Nc = c->mbl_Nc;
    L.chars_sys = cs;
    L.spec_div = c->spec_div;
    if (!words.empty()) {
        L.words = upload(h, words);
        if (!L.words) return fail(h, QJX_ERR_OOM, "MBL words");
    }
    CK(cudaMemsetAsync(L.var_pos, 0, n * sizeof(long long), h->stream));
    CK(cudaMemsetAsync(L.ratio, 0, n * sizeof(double), h->stream));
    CK(cudaMemsetAsync(L.ds_rec, 0, n * sizeof(double), h->stream));
    CK(cudaMemsetAsync(L.df_rec, 0, n * sizeof(double), h->stream));
    CK(cudaMemsetAsync(L.eps_iters, 0, n * sizeof(int), h->stream));
    CK(cudaMemsetAsync(L.eps, 0, n * sizeof(double), h->stream));
    CK(launch_lpn(P, L, 0, 0.0, -1, h->stream));
    h->stats.launches += 1;
    CK(cudaStreamSynchronize(h->stream));
    h->lpn_started = true;
    return QJX_OK;
}

extern "C" qjx_status qjx_lpn_bases(qjx_engine *h)
{
    NvtxRange range("qjx_lpn_bases");
    if (!h) return QJX_ERR_INVALID_ARG;
    if (!h->lpn_started) return fail(h, QJX_ERR_STATE, "qjx_lpn_start first");
    CK(cudaSetDevice(h->cfg.device));
    CK(launch_lpn(h->P, h->L, 2, 0.0, -1, h->stream));
    h->stats.launches += 1;
    CK(cudaStreamSynchronize(h->stream));
    return QJX_OK;
}

extern "C" qjx_status qjx_lpn_period(qjx_engine *h, double curr_time, int adr_dump)
{
    NvtxRange range("qjx_lpn_period");
    if (!h) return QJX_ERR_INVALID_ARG;
    if (!h->lpn_started) return fail(h, QJX_ERR_STATE, "qjx_lpn_start first");
    if (adr_dump < -1 || adr_dump >= h->cfg.max_dumps) return fail(h, QJX_ERR_INVALID_ARG, "adr_dump out of range");
    CK(cudaSetDevice(h->cfg.device));
    CK(launch_lpn(h->P, h->L, 1, curr_time, adr_dump, h->stream));
    h->stats.launches += 1;
    CK(cudaStreamSynchronize(h->stream));
    return QJX_OK;
}

extern "C" qjx_status qjx_lpn_get(qjx_engine *h, double *lambda_now, double *lambda, double *delta_s,
                                  double *mean_lpn, double *energy_lpn, double *robs_lpn, int *num_renorms)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    if (!h->lpn_started) return fail(h, QJX_ERR_STATE, "qjx_lpn_start first");
    CK(cudaSetDevice(h->cfg.device));
    const LpnParams &L = h->L;
    const size_t n = h->P.n;
    if (lambda_now) CK(cudaMemcpy(lambda_now, L.lambda_now, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (lambda) CK(cudaMemcpy(lambda, L.lambda, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (delta_s) CK(cudaMemcpy(delta_s, L.delta_s_v, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (mean_lpn) CK(cudaMemcpy(mean_lpn, L.mean_lpn, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (energy_lpn) CK(cudaMemcpy(energy_lpn, L.energy_lpn, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (robs_lpn && h->P.nr > 0)
        CK(cudaMemcpy(robs_lpn, L.robs_lpn, n * h->P.nr * sizeof(double2), cudaMemcpyDeviceToHost));
    if (num_renorms) CK(cudaMemcpy(num_renorms, L.num_renorms, n * sizeof(int), cudaMemcpyDeviceToHost));
    return QJX_OK;
}

extern "C" qjx_status qjx_lpn_get_last(qjx_engine *h, int *renormed, double *ratio, double *delta_s,
                                       double *delta_f, int *eps_iters, double *eps)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    if (!h->lpn_started) return fail(h, QJX_ERR_STATE, "qjx_lpn_start first");
    CK(cudaSetDevice(h->cfg.device));
    const LpnParams &L = h->L;
    const size_t n = h->P.n;
    if (renormed) CK(cudaMemcpy(renormed, L.renormed, n * sizeof(int), cudaMemcpyDeviceToHost));
    if (ratio) CK(cudaMemcpy(ratio, L.ratio, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (delta_s) CK(cudaMemcpy(delta_s, L.ds_rec, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (delta_f) CK(cudaMemcpy(delta_f, L.df_rec, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (eps_iters) CK(cudaMemcpy(eps_iters, L.eps_iters, n * sizeof(int), cudaMemcpyDeviceToHost));
    if (eps) CK(cudaMemcpy(eps, L.eps, n * sizeof(double), cudaMemcpyDeviceToHost));
    return QJX_OK;
}

// ---------------------------------------------------------------- checkpoint / resume
namespace {
struct CkptHeader {
    uint64_t magic;  // 'QJXCKPT1'
    int n, MD, slots, nd, E, lpn, nr, period_base;
};
constexpr uint64_t kCkptMagic = 0x3154504b43584a51ULL;

// (device pointer, bytes) of every array a checkpoint carries, in blob order
std::vector<std::pair<void *, size_t>> ckpt_parts(qjx_engine *h)
{
    const Params &P = h->P;
    const size_t n = P.n;
    const int slots = P.prop == 1 ? kRkSlots : 2;
    std::vector<std::pair<void *, size_t>> v = {
        {P.psi, (size_t)slots * n * P.MD * sizeof(double2)},
        {P.st, n * sizeof(TrajState)},
        {P.gn, n * P.nd * sizeof(double)},
        {P.mean_start, n * sizeof(double)},
    };
    if (h->lpn_alloc) {
        const LpnParams &L = h->L;
        v.push_back({L.lambda, n * sizeof(double)});
        v.push_back({L.lambda_now, n * sizeof(double)});
        v.push_back({L.delta_s_v, n * sizeof(double)});
        v.push_back({L.mean_lpn, n * sizeof(double)});
        v.push_back({L.energy_lpn, n * sizeof(double)});
        v.push_back({L.robs_lpn, n * std::max(1, P.nr) * sizeof(double2)});
        v.push_back({L.num_renorms, n * sizeof(int)});
        v.push_back({L.var_pos, n * sizeof(long long)});
    }
    if (h->d_active) v.push_back({h->d_active, n});
    return v;
}
}  // namespace

extern "C" qjx_status qjx_checkpoint_size(qjx_engine *h, size_t *bytes)
{
    if (!h || !bytes) return QJX_ERR_INVALID_ARG;
    size_t b = sizeof(CkptHeader);
    for (const auto &p : ckpt_parts(h)) b += p.second;
    *bytes = b;
    return QJX_OK;
}

extern "C" qjx_status qjx_checkpoint_save(qjx_engine *h, void *buf, size_t bytes)
{
    size_t need = 0;
    if (!h || !buf || qjx_checkpoint_size(h, &need) != QJX_OK || bytes < need) return QJX_ERR_INVALID_ARG;
    if (!h->states_set) return fail(h, QJX_ERR_STATE, "nothing to checkpoint: qjx_set_states first");
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaStreamSynchronize(h->stream));
    const Params &P = h->P;
    CkptHeader hd{kCkptMagic, P.n, P.MD, P.prop == 1 ? kRkSlots : 2, P.nd, P.E, h->lpn_alloc ? 1 : 0, P.nr,
                  h->period_base};
    unsigned char *o = static_cast<unsigned char *>(buf);
    std::memcpy(o, &hd, sizeof(hd));
    o += sizeof(hd);
    for (const auto &p : ckpt_parts(h)) {
        CK(cudaMemcpy(o, p.first, p.second, cudaMemcpyDeviceToHost));
        o += p.second;
    }
    return QJX_OK;
}

extern "C" qjx_status qjx_checkpoint_load(qjx_engine *h, const void *buf, size_t bytes)
{
    if (!h || !buf || bytes < sizeof(CkptHeader)) return QJX_ERR_INVALID_ARG;
    CkptHeader hd;
    std::memcpy(&hd, buf, sizeof(hd));
    const Params &P = h->P;
    if (hd.magic != kCkptMagic || hd.n != P.n || hd.MD != P.MD || hd.slots != (P.prop == 1 ? kRkSlots : 2) ||
        hd.nd != P.nd || hd.E != P.E || hd.nr != P.nr)
        return fail(h, QJX_ERR_INVALID_ARG, "checkpoint of a different engine configuration");
    if (hd.lpn && !h->lpn_alloc)
        return fail(h, QJX_ERR_STATE, "checkpoint carries the Lyapunov task: qjx_lpn_start this engine first");
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaStreamSynchronize(h->stream));
    const unsigned char *in = static_cast<const unsigned char *>(buf) + sizeof(hd);
    const unsigned char *end = static_cast<const unsigned char *>(buf) + bytes;
    for (const auto &p : ckpt_parts(h)) {
        const bool lpn_part = h->lpn_alloc && (p.first == h->L.lambda || p.first == h->L.lambda_now ||
                                               p.first == h->L.delta_s_v || p.first == h->L.mean_lpn ||
                                               p.first == h->L.energy_lpn || p.first == h->L.robs_lpn ||
                                               p.first == h->L.num_renorms || p.first == h->L.var_pos);
        if (lpn_part && !hd.lpn) continue;
        if (in + p.second > end) return fail(h, QJX_ERR_INVALID_ARG, "truncated checkpoint");
        CK(cudaMemcpy(p.first, in, p.second, cudaMemcpyHostToDevice));
        in += p.second;
    }
    h->period_base = hd.period_base;
    h->states_set = true;
    if (hd.lpn) h->lpn_started = true;
    for (int i = 0; i < P.n; i++) {
        h->jt[i].clear();
        h->jn[i].clear();
        h->je[i].clear();
        h->jtype[i].clear();
    }
    return QJX_OK;
}

extern "C" qjx_status qjx_set_trace(qjx_engine *h, int enable)
{
    if (!h) return QJX_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->cfg.device));
    if (enable && !h->P.trace) {
        h->P.trace = (long long *)dalloc(h, (size_t)h->grid * kTraceFields * sizeof(long long));
        if (!h->P.trace) return QJX_ERR_OOM;
    } else if (enable) {
        CK(cudaMemset(h->P.trace, 0, (size_t)h->grid * kTraceFields * sizeof(long long)));
    } else {
        h->P.trace = nullptr;  // buffer stays owned by the engine until qjx_destroy
    }
    return QJX_OK;
}

extern "C" qjx_status qjx_get_trace(qjx_engine *h, int64_t *out, int *n_ctas, int *n_fields)
{
    if (!h || !n_ctas || !n_fields) return QJX_ERR_INVALID_ARG;
    *n_ctas = h->grid;
    *n_fields = kTraceFields;
    if (!h->P.trace || !out) return h->P.trace ? QJX_OK : QJX_ERR_STATE;
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaMemcpy(out, h->P.trace, (size_t)h->grid * kTraceFields * sizeof(long long), cudaMemcpyDeviceToHost));
    return QJX_OK;
}

extern "C" qjx_status qjx_measure_fp64_peak(int device, double *ffma_tflops, double *dmma_tflops)
{
    if (!ffma_tflops && !dmma_tflops) return QJX_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return QJX_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *out = nullptr;
    if (cudaMalloc(&out, 16) != cudaSuccess) return QJX_ERR_OOM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 4, iters = 1 << 16;
    double best = 0.0, best_mma = 0.0;
    for (int r = 0; r < 6; r++) {  // first round of each is a warm-up
        cudaEventRecord(a, 0);
        launch_fp64_peak(out, blocks, iters, 0);
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        const double fl = 2.0 * 8.0 * (double)iters * blocks * 256.0;  // 8 fma chains per thread
        if (r) best = std::max(best, fl / (ms * 1e-3) / 1e12);
        cudaEventRecord(a, 0);
        launch_dmma_peak(out, blocks, iters / 4, 0);
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        const double fm = 512.0 * 8.0 * (double)(iters / 4) * blocks * 8.0;  // 8 mma chains per warp
        if (r) best_mma = std::max(best_mma, fm / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess) return QJX_ERR_CUDA;
    if (ffma_tflops) *ffma_tflops = best;
    if (dmma_tflops) *dmma_tflops = best_mma;
    return QJX_OK;
}

// ---------------------------------------------------------------- autotuner
extern "C" qjx_status qjx_autotune(const qjx_config *cfg, const double *U, const double *L, const double *g,
                                   const double *HE, int n_periods, qjx_tiles *best, qjx_tiles *cand, double *us,
                                   int *n_cand)
{
    if (!cfg || !U || !L || !g || !HE || !best || n_periods < 1 || ((cand || us) && !n_cand))
        return QJX_ERR_INVALID_ARG;
    const int d = cfg->d, n = cfg->n_traj;
    if (d < 2 || n < 1) return QJX_ERR_INVALID_ARG;
    std::vector<qjx_tiles> list;
    if (cfg->precision == 1) {
        for (int st : {2, 3, 4, 6, 8})
            for (int rows : {8, 32, 64, 128}) list.push_back(qjx_tiles{0, 0, st, rows});
    } else {
        for (int nc : {32, 16, 8})
            for (int kb : {16, 12, 8, 4}) list.push_back(qjx_tiles{nc, kb, 0, 0});
    }
    std::vector<double> psi((size_t)n * d * 2, 0.0);
    for (int i = 0; i < n; i++) psi[(size_t)i * d * 2] = 1.0;  // |0>
    const int cap = n_cand ? *n_cand : 0;
    int filled = 0;
    double best_us = 0.0;
    for (const qjx_tiles &t : list) {
        qjx_config c = *cfg;
        c.tiles = t;
        c.num_robs = 0;
        c.record = 0;
        c.max_dumps = 1;
        qjx_engine *h = nullptr;
        if (create_engine(&c, U, L, g, HE, nullptr, 2, &h) != QJX_OK) continue;  // the shape does not fit
        double t_us = -1.0;
        if (qjx_set_states(h, psi.data()) == QJX_OK && qjx_init_thresholds(h) == QJX_OK &&
            qjx_run_periods(h, 1, 0, nullptr, 0, 0) == QJX_OK) {
            const double ms0 = h->stats.step_kernel_ms;
            if (qjx_run_periods(h, n_periods, 0, nullptr, 0, 0) == QJX_OK)
                t_us = (h->stats.step_kernel_ms - ms0) * 1e3 / ((double)n * n_periods);
        }
        qjx_destroy(h);
        if (t_us <= 0.0) continue;
        if (filled < cap) {
            if (cand) cand[filled] = t;
            if (us) us[filled] = t_us;
            filled++;
        }
        if (best_us == 0.0 || t_us < best_us) {
            best_us = t_us;
            *best = t;
        }
    }
    if (n_cand) *n_cand = filled;
    if (best_us == 0.0) return QJX_ERR_UNSUPPORTED;
    tile_cache_put(cfg->precision, d, *best, best_us);
    return QJX_OK;
}

extern "C" qjx_status qjx_mem_info(int device, size_t *free_bytes, size_t *total_bytes)
{
    if (!free_bytes || !total_bytes) return QJX_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return QJX_ERR_CUDA;
    return cudaMemGetInfo(free_bytes, total_bytes) == cudaSuccess ? QJX_OK : QJX_ERR_CUDA;
}

extern "C" qjx_status qjx_engine_bytes(qjx_engine *h, size_t *bytes)
{
    if (!h || !bytes) return QJX_ERR_INVALID_ARG;
    *bytes = h->dev_bytes;
    return QJX_OK;
}
