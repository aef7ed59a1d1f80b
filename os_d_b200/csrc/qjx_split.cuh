// qjx_split.cuh -- the split-precision micro-step on the tcgen05 tensor cores (precision 1).
//
// Same lock-step micro-steps, buckets and trajectory state machine as the FP64 plain form;
// only the d x d complex matvec changes.  Roles are transposed against the FP64 kernel so that
// the trajectory, not the matrix row, is the MMA M dimension, and the complex product is four
// real GEMMs sharing operands:
//
//   Re y[m][r] = sum_k Xr[m][k] Ur[r][k] - Xi[m][k] Ui[r][k]     m: trajectory (128 TMEM lanes)
//   Im y[m][r] = sum_k Xr[m][k] Ui[r][k] + Xi[m][k] Ur[r][k]     r: output row (MMA N = MDs)
//
//   A = the tile's states (Xr, Xi) as bf16 planes, written by the CTA from the FP64 states,
//   B = Re M and Im M as bf16 planes prepared once by the host,
//   D = two FP32 accumulators in tensor memory, Re in columns [0, MDs), Im in [MDs, 2 MDs);
//       the minus sign is the instruction descriptor's negate-A bit.
//
// Every operand x is split x = hi + lo with hi = bf16(x), lo = bf16(x - hi); the MMAs add
// hi*hi + hi*lo + lo*hi in FP32 ("bf16x3"), which leaves about 2^-16 of relative error per
// product and the FP32 accumulation error (measured about 4e-6 of max|y| per matvec at
// d = 201).  The accumulators are read back to FP64 and the FP64 epilogue of the plain form
// runs unchanged (norm test, jump, renormalisation, observables), except that a norm within the
// split error of the threshold is not decided: that trajectory's step is computed again as an
// FP64 matvec (the plain form's arithmetic) by a CTA the split tiles leave free, which decides.
//
// Shared-memory operands use the K-major no-swizzle canonical layout: a core matrix is
// 8 rows x 16 bytes (8 bf16 along K) stored contiguously; within one k-step (16 bf16 of K)
// the two K-halves of a row group are 128 bytes apart (leading byte offset) and consecutive
// 8-row groups 256 bytes apart (stride byte offset).  The host writes B in exactly this
// order, so one k-step of all four B planes is one contiguous TMA bulk copy.
//
// Per tile (one matrix, up to 128 trajectories of one bucket) a ring of S stages, one k-step of
// A and B planes each:
//   warps 0-3, 6-9, 10-13   three producer groups; group p converts the k-steps ks = p (mod 3):
//               FP64 state -> bf16 planes of A (a warp-wide 256-bit load covers 8 rows x 128 bytes;
//               generic stores, then fence.proxy.async and an arrive on fullA)
//   warp 4      one thread issues the bulk copy of the B planes (complete_tx on fullB)
//   warp 5      one thread issues the 12 tcgen05.mma of a k-step and commits them to empty[stage]
//   warps 14-15 load the tile's trajectory records meanwhile
// then the FP32 accumulators of up to 64 trajectories at a time are staged in the idle ring by
// the warps that own their TMEM lane quarters, and every warp runs its trajectories through the
// epilogue and appends them to their next buckets.  A batched engine's ensembles each have their
// own padded rows and k-steps; the tile plan of the next micro-step (rows per tile, first tile of
// every bucket) is made by the last CTA to finish one.  One cooperative launch runs a batch of
// micro-steps: between two of them every CTA waits at a grid barrier (an arrival counter, and a
// generation number the planning CTA releases), and the operand ring, mbarriers and tensor
// memory stay set up across them.

constexpr int kAPlanes = 4;                  // A and B planes: Re hi, Re lo, Im hi, Im lo
constexpr int kTileM = 128;                  // MMA M = TMEM lanes (a tile holds up to 128 trajectories)
constexpr int kMaxSStages = kMaxSplitStages;  // operand ring depth (runtime: the tile shape's, at most this)
constexpr int kABytes = kTileM * 32;         // one plane of one k-step of A: 128 rows x 16 bf16
constexpr int kTmemCols = 512;
constexpr long long kSplitWait = 1ll << 20;  // bounded mbarrier polls (normal waits end within microseconds)
constexpr long long kGridWait = 1ll << 24;   // bounded polls of the grid barrier (a micro-step is ~50 us)

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu)        // start address
           | ((uint64_t)(128u >> 4) << 16)           // leading byte offset: K-half stride
           | ((uint64_t)(256u >> 4) << 32)           // stride byte offset: 8-row group stride
           | (1ull << 46);                           // descriptor version of sm_100
}

// kind::f16 instruction descriptor: FP32 accumulator, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 8 consecutive FP32 accumulator columns of this thread's TMEM lane at each of two addresses (the
// Re and Im accumulators), both loads in flight before the one wait.
__device__ __forceinline__ void tmem_ld8x2(uint32_t ta, uint32_t tb, float *va, float *vb)
{
    uint32_t a[8], b[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7])
                 : "r"(ta));
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7])
                 : "r"(tb));
    // the registers are valid after wait::ld; tying them to the wait keeps every use behind it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]),
                   "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]), "+r"(b[7])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) {
        va[i] = __uint_as_float(a[i]);
        vb[i] = __uint_as_float(b[i]);
    }
}

// Two consecutive complex components (32 bytes, 32-byte aligned) in one 256-bit load, cached in L2
// only: the state rows stream through once, and in L1 they would evict the small per-ensemble
// tables that every trajectory's epilogue reads.
__device__ __forceinline__ void ld_pair(const double2 *p, double2 &a, double2 &b)
{
    asm volatile("ld.global.cg.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
                 : "l"(p));
}

// hi/lo planes of one (re, im) pair packed as two bf16 (re in the low half: lower address):
// hi = bf16(f), lo = bf16(f - hi) with f the FP32 rounding of the FP64 value (f - hi is exact in
// FP32; the FP32 rounding, 2^-24, is far below the 2^-17 the two planes resolve).
__device__ __forceinline__ void split_pair(double2 v, uint32_t &hi, uint32_t &lo)
{
    const float fr = __double2float_rn(v.x), fi = __double2float_rn(v.y);
    const __nv_bfloat162 h = __floats2bfloat162_rn(fr, fi);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(fr - hf.x, fi - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

// FP64 recheck of one trajectory's step: y = M x with the plain form's arithmetic (per output the
// k-ascending fma chain of the contract, k up to the even kp), the matrix streamed through the free
// operand ring in slabs of kb k rows by TMA bulk copies (two buffers, mbarriers rbar[0..1]), then
// the epilogue decides with the FP64 norm and the trajectory joins its next bucket.  Whole CTA;
// returns false when a bounded wait gave up.
__device__ bool recheck_column(const Params &P, int tr, unsigned char *smem, TrajState *st_s, uint64_t *rbar,
                               uint32_t &rphase, int *cnt_next, int *list_next)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) load_state(st_s, &P.st[tr]);
    __syncthreads();
    const TrajState st = *st_s;
    const int dg = P.e_d[st.ens], MDg = 8 * ((dg + 7) / 8), kp = (dg + 1) & ~1, kb = P.rchk_kb;
    const int g = P.e_g0[st.ens] + st.b * P.deep + st.lvl;
    const double2 *mat = P.mats + P.g_off[g];
    double2 *slab = reinterpret_cast<double2 *>(smem);  // [2][kb][MDg]
    double2 *xs = slab + 2 * (size_t)kb * MDg;           // [kp] input
    double2 *ys = xs + kp;                               // [MDg] FP64 product
    const double2 *x = slot_ptr(P, st.cur, tr);
    for (int k = tid; k < kp; k += blockDim.x) xs[k] = (k < dg) ? x[k] : make_double2(0.0, 0.0);
    const int nslab = (kp + kb - 1) / kb;
    if (tid == 0) {
        fence_proxy_async();
        for (int q = 0; q < 2 && q < nslab; q++) {
            const int kc = min(kb, kp - q * kb);
            mbar_expect_tx(&rbar[q], (uint32_t)(kc * MDg * 16));
            bulk_g2s(slab + (size_t)q * kb * MDg, mat + (size_t)q * kb * MDg, (uint32_t)(kc * MDg * 16), &rbar[q]);
        }
    }
    __syncthreads();
    bool ok = true;
    double re = 0.0, im = 0.0;
    for (int sl = 0; sl < nslab; sl++) {
        const int q = sl & 1;
        if (!mbar_wait_bounded(&rbar[q], (rphase >> q) & 1u, kSplitWait)) ok = false;
        rphase ^= 1u << q;
        const int k0 = sl * kb, kc = min(kb, kp - k0);
        if (ok && tid < dg) {
            const double2 *Mq = slab + (size_t)q * kb * MDg + tid;
            for (int kk = 0; kk < kc; kk++) {
                const double2 m = Mq[(size_t)kk * MDg], v = xs[k0 + kk];
                re = __fma_rn(m.x, v.x, re);
                re = __fma_rn(-m.y, v.y, re);
                im = __fma_rn(m.x, v.y, im);
                im = __fma_rn(m.y, v.x, im);
            }
        }
        __syncthreads();
        if (tid == 0 && ok && sl + 2 < nslab) {
            const int kn = min(kb, kp - (sl + 2) * kb);
            fence_proxy_async();
            mbar_expect_tx(&rbar[q], (uint32_t)(kn * MDg * 16));
            bulk_g2s(slab + (size_t)q * kb * MDg, mat + (size_t)(sl + 2) * kb * MDg, (uint32_t)(kn * MDg * 16), &rbar[q]);
        }
    }
    if (!__syncthreads_and(ok ? 1 : 0)) return false;
    if (tid < dg) ys[tid] = make_double2(re, im);
    __syncthreads();
    if (warp == 0) {
        const int g2 = column_epilogue(P, ys, tr, st, lane);
        if (g2 >= 0 && lane == 0) {
            const int pos = atomicAdd(&cnt_next[g2], 1);
            list_next[P.g_loff[g2] + pos] = tr;
        }
    }
    fence_proxy_async();  // generic writes to the ring before later bulk copies into it
    __syncthreads();
    return true;
}

// Tile plan of a micro-step from its bucket sizes cnt[G] and its rtot FP64 rechecks (block-wide,
// blockDim.x a multiple of 32): rows per tile R, the smallest multiple of 8 (at least P.min_rows,
// at most 128) whose tiles fit one wave of `grid` CTAs next to the rechecks, so that trajectories
// and their epilogues spread over all SMs; then the first tile of every group.
// Rows per tile of a bucket when the plan's rows per tile is R: when the tiles fit one wave, the
// jump-operator and observable buckets take about 5/8 of R (their epilogues renormalise, draw and
// reduce: a tile of them took 1.3x as long as a matrix bucket's tile of as many rows, and a
// micro-step waits for its slowest tile); the (branch, level) buckets, and every bucket when the
// tiles take several waves (a batch of many ensembles: more tiles would only add MMA work), R.
__device__ __forceinline__ bool heavy_group(const Params &P, int g)
{
    return g - P.e_g0[P.g_ens[g]] >= P.nb * P.deep;
}
__device__ __forceinline__ int group_rows(int R, bool heavy) { return heavy ? max(8, (R * 5 / 8) & ~7) : R; }

__device__ void split_plan(const Params &P, const int *cnt, int rtot, int grid)
{
    __shared__ int w_t[32][17];
    __shared__ int w_s[32];
    __shared__ int s_R, s_hv;
    const int G = P.G, nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    int part[16];
#pragma unroll
    for (int j = 0; j < 16; j++) part[j] = 0;
    for (int g = tid; g < G; g += nt) {
        const int m = __ldcg(cnt + g);
        const bool hv = heavy_group(P, g);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int r = group_rows(8 * j + 8, hv);
            part[j] += (m + r - 1) / r;
        }
    }
#pragma unroll
    for (int j = 0; j < 16; j++) {
        int v = part[j];
        for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) w_t[warp][j] = v;
    }
    __syncthreads();
    if (tid == 0) {
        const int avail = max(1, grid - rtot);
        int R = kTileM, hv = 0;
        for (int j = 0; j < 16; j++) {
            int tiles = 0;
            for (int w = 0; w < nw; w++) tiles += w_t[w][j];
            if (tiles <= avail) {
                R = 8 * (j + 1);
                hv = 1;
                break;
            }
        }
        s_R = max(P.min_rows, R);
        s_hv = hv;
    }
    __syncthreads();
    const int R = s_R;
    const bool hv = s_hv != 0;
    // exclusive scan of the tiles per group over the block: each thread a contiguous range
    const int per = (G + nt - 1) / nt, g0 = min(G, tid * per), g1 = min(G, g0 + per);
    int c = 0;
    for (int g = g0; g < g1; g++) {
        const int r = group_rows(R, hv && heavy_group(P, g));
        c += (__ldcg(cnt + g) + r - 1) / r;
    }
    int inc = c;
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
    }
    if (lane == 31) w_s[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int v = lane < nw ? w_s[lane] : 0;
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v += y;
        }
        if (lane < nw) w_s[lane] = v;
    }
    __syncthreads();
    int acc = inc - c + (warp ? w_s[warp - 1] : 0);
    for (int g = g0; g < g1; g++) {
        P.splan[1 + g] = acc;
        const int r = group_rows(R, hv && heavy_group(P, g));
        acc += (__ldcg(cnt + g) + r - 1) / r;
    }
    if (tid == nt - 1) {
        P.splan[1 + G] = acc;
        P.splan[0] = R | (hv ? 0x10000 : 0);  // rows per tile; the bit: heavy buckets take fewer
    }
    __syncthreads();
}

// Plan of step 0 after a host-side enqueue (one block).
__global__ void __launch_bounds__(512) split_plan_kernel(const Params P, int grid)
{
    split_plan(P, P.cnt, __ldcg(P.rcnt), grid);
}

// Group of tile t: the last g with splan[1 + g] <= t (warp-cooperative search over the global plan).
__device__ __forceinline__ int split_tile_group(const Params &P, int t, int lane)
{
    int lo = 0, hi = P.G;  // answer in [lo, hi)
    while (hi - lo > 1) {
        const int step = (hi - lo + 31) / 32;
        const int g = lo + lane * step;
        const bool le = g < hi && __ldcg(P.splan + 1 + g) <= t;
        const unsigned m = __ballot_sync(0xffffffffu, le);
        const int last = 31 - __clz(m);  // lane 0 always qualifies (splan[1 + lo] <= t)
        lo = lo + last * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// Dynamic shared memory: a ring of `stages` operand stages, each [A planes][B planes] of one
// k-step; after the MMAs of a tile the ring holds the epilogue's FP32 accumulators of up to 64
// trajectories (one row of 2 MDs + 1 floats each: Re then Im) and one FP64 column per warp.
size_t split_stage_bytes(int MDs) { return (size_t)kAPlanes * (kABytes + (size_t)MDs * 32); }

__host__ __device__ inline size_t split_epi_f32_bytes(int MDs, int rows)
{
    return ((size_t)rows * (2 * MDs + 1) * 4 + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t split_epi_bytes(int MDs, int rows)
{
    return split_epi_f32_bytes(MDs, rows) + (size_t)(kThreads / 32) * (MDs + 1) * sizeof(double2);
}

size_t split_smem_bytes(int MDs, int MD, int stages)
{
    const size_t ring = (size_t)stages * split_stage_bytes(MDs);
    (void)MD;
    const size_t epi = split_epi_bytes(MDs, 32);
    return ring > epi ? ring : epi;
}

__global__ void __launch_bounds__(kThreads, 1) split_step_kernel(const Params P, int s0, int nsteps)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = P.sstages;
    const size_t stage_bytes = (size_t)kAPlanes * (kABytes + (size_t)P.MDs * 32);  // ring stride (largest MDs)
    __shared__ __align__(8) uint64_t fullA[kMaxSStages], fullB[kMaxSStages], empty[kMaxSStages], accf, rbar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_tr[kTileM];
    __shared__ long long s_src[kTileM];
    __shared__ __align__(16) TrajState s_st[kTileM];
    __shared__ int s_fail, s_last;
    __shared__ unsigned int s_gen;
    __shared__ int w_g2[kThreads / 32][kTileM / (kThreads / 32)];  // per warp: its trajectories' next buckets

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // epilogue rows staged per pass: 64 when their FP32 accumulators and the warps' FP64 columns
    // fit the dynamic shared memory, else 32
    const size_t dyn = max((size_t)S * stage_bytes, split_epi_bytes(P.MDs, 32));
    const int RP = split_epi_bytes(P.MDs, 64) <= dyn ? 64 : 32;
    double2 *wcol = reinterpret_cast<double2 *>(smem + split_epi_f32_bytes(P.MDs, RP)) + (size_t)warp * (P.MDs + 1);
    const int G = P.G, n = P.n;
    if (warp == 0) {
        if (lane == 0) {
            for (int q = 0; q < S; q++) {
                mbar_init(&fullA[q], kTileM);
                mbar_init(&fullB[q], 1);
                mbar_init(&empty[q], 1);
            }
            mbar_init(&accf, 1);
            mbar_init(&rbar[0], 1);
            mbar_init(&rbar[1], 1);
            s_fail = 0;
            fence_proxy_async();
        }
        __syncwarp();
        // the whole tensor memory of the SM (one CTA per SM)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"((uint32_t)kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    long long work = 0, nrechk = 0;
    uint32_t ntile = 0, kit = 0, rphase = 0;  // tiles done, k-steps issued (ring position)
    bool ok = true;
    long long tr_setup = 0, tr_mma = 0, tr_stage = 0, tr_epi = 0;
    const long long t_begin = clock64();
    int steps_done = 0;

    // micro-steps s0 .. s0 + nsteps - 1 (one, when launched per step); between two steps of one
    // launch every CTA waits at a grid barrier whose last arrival plans the next step
    for (int si = 0; si < nsteps; si++) {
        const int s = s0 + si;
        const int *cnt_cur = P.cnt + (s % 3) * G;
        int *cnt_next = P.cnt + ((s + 1) % 3) * G;
        const int *list_cur = P.lists + (size_t)(s & 1) * P.ltot;
        int *list_next = P.lists + (size_t)((s + 1) & 1) * P.ltot;
        const int *rlist_cur = P.rlist + (size_t)(s & 1) * P.n;
        int *rlist_next = P.rlist + (size_t)((s + 1) & 1) * P.n;
        int *rcnt_next = P.rcnt + (s + 1) % 3;
        const int Rtot = __ldcg(P.rcnt + s % 3);  // FP64 rechecks of this micro-step
        const int Rw = __ldcg(P.splan), T = __ldcg(P.splan + 1 + G);  // this step's plan (rows per tile, tiles)
        const int R = Rw & 0xFFFF;
        const bool heavy_fewer = (Rw >> 16) != 0;
        if (T + Rtot == 0) break;  // nothing left in this call (every CTA reads the same plan)
        if (blockIdx.x == 0) {
            for (int i = tid; i < G; i += kThreads) P.cnt[((s + 2) % 3) * G + i] = 0;
            if (tid == 0) P.rcnt[(s + 2) % 3] = 0;
        }

        for (int t = blockIdx.x; t < T + Rtot && ok; t += gridDim.x) {
            if (t >= T) {  // an FP64 recheck (the CTAs past the split tiles take these first)
                if (!recheck_column(P, rlist_cur[t - T], smem, &s_st[0], rbar, rphase, cnt_next, list_next)) {
                    ok = false;
                    break;
                }
                work += 1;
                nrechk += 1;
                continue;
            }
            const long long t0 = clock64();
            const int g = split_tile_group(P, t, lane);  // every warp finds it (warp-uniform)
            const int e = P.g_ens[g];
            const int d = P.e_d[e], MDs = P.e_mds[e], KS = P.e_ks[e], bbytes = MDs * 32;
            const int Rg = group_rows(R, heavy_fewer && g - P.e_g0[e] >= P.nb * P.deep);
            const int base = (t - __ldcg(P.splan + 1 + g)) * Rg;
            const int rows = min(Rg, __ldcg(cnt_cur + g) - base);
            if (tid < kTileM) {
                if (tid < rows) {
                    const int tr = list_cur[P.g_loff[g] + base + tid];
                    const TrajState *sp = &P.st[tr];
                    const int slot = src_slot(sp->phase, sp->cur, sp->rk_stage);
                    s_tr[tid] = tr;
                    s_src[tid] = ((long long)slot * n + tr) * P.MD;
                } else {
                    s_tr[tid] = -1;
                    s_src[tid] = -1;
                }
            }
            __syncthreads();
            const long long t1 = clock64();
            const uint32_t it0 = kit;  // k-steps issued before this tile
            const uint32_t idesc = umma_idesc_bf16(kTileM, MDs);
            const uint32_t idesc_neg = idesc | (1u << 13);  // negate A

            const int agrp = (warp < 4) ? 0 : (warp >= 6 && warp < 10) ? 1 : (warp >= 10 && warp < 14) ? 2 : -1;
            if (agrp >= 0) {
                // A producers: group p (4 warps) handles the k-steps ks = p (mod 3), so three
                // independent load-convert chains run in parallel.  One warp-wide load covers 8 rows x
                // one K-half (components 16 ks + 8 hh .. + 7, 128 contiguous bytes of each row): lane l
                // takes row 8 rb + l / 4 and the component pair 2 (l % 4), 2 (l % 4) + 1, so every
                // 32-byte sector is read whole by one lane, and a round's four plane stores are 128
                // contiguous bytes each.  Round u of a warp is the (row block, half) pair 4 u + warp;
                // all rounds of a k-step are loaded before the stage is waited for.  Rows past the
                // tile's last trajectory are neither loaded nor stored: row i of an accumulator depends
                // on row i of A only, and the epilogue reads live rows only.
                const int gw = warp - (agrp == 0 ? 0 : (agrp == 1 ? 6 : 10));
                const int r8 = lane >> 2, jq = lane & 3;
                const int npairs = 2 * ((rows + 7) >> 3);
                for (int ks = agrp; ks < KS && ok; ks += 3) {
                    const uint32_t it = it0 + ks, q = it % S;
                    unsigned char *As = smem + q * stage_bytes + 4 * lane;
                    for (int u0 = 0; u0 < 8; u0 += 4) {
                        if (u0 > 0 && 4 * u0 + gw >= npairs) break;  // warp-uniform
                        double2 v[4][2];
    #pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const int pi = 4 * (u0 + u) + gw, m = 8 * (pi >> 1) + r8;
                            const int k = 16 * ks + 8 * (pi & 1) + 2 * jq;
                            // every lane of a live round loads (a lane without data reads component 0
                            // of row 0) and nothing touches v before the stage wait, so the four loads
                            // are in flight together: a select or a write on a load's destination
                            // registers would wait for that load.  k + 1 < MD: inside the row.
                            const long long so = (m < rows && k < d) ? s_src[m] + k : 0;
                            if (pi < npairs) ld_pair(P.psi + so, v[u][0], v[u][1]);
                        }
                        if (u0 == 0 && it >= (uint32_t)S && !mbar_wait_bounded(&empty[q], ((it / S) - 1) & 1u, kSplitWait))
                            ok = false;
    #pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const int pi = 4 * (u0 + u) + gw, m = 8 * (pi >> 1) + r8;
                            if (pi >= npairs || m >= rows) continue;
                            // components from d on are row padding (or were not loaded): zeros
                            const int k = 16 * ks + 8 * (pi & 1) + 2 * jq;
                            const double2 z = make_double2(0.0, 0.0);
                            const double2 a = (k < d) ? v[u][0] : z, b = (k + 1 < d) ? v[u][1] : z;
                            uint32_t rh, rl, ih, il;
                            split_pair(make_double2(a.x, b.x), rh, rl);
                            split_pair(make_double2(a.y, b.y), ih, il);
                            unsigned char *dst = As + 256 * (pi >> 1) + 128 * (pi & 1);
                            *reinterpret_cast<uint32_t *>(dst) = rh;
                            *reinterpret_cast<uint32_t *>(dst + kABytes) = rl;
                            *reinterpret_cast<uint32_t *>(dst + 2 * kABytes) = ih;
                            *reinterpret_cast<uint32_t *>(dst + 3 * kABytes) = il;
                        }
                    }
                    fence_proxy_async();
                    mbar_arrive(&fullA[q]);
                }
            } else if (warp == 4) {
                if (lane == 0) {  // B producer
                    const unsigned char *ug = P.usplit + P.g_uoff[g];
                    for (int ks = 0; ks < KS && ok; ks++) {
                        const uint32_t it = it0 + ks, q = it % S;
                        if (it >= (uint32_t)S && !mbar_wait_bounded(&empty[q], ((it / S) - 1) & 1u, kSplitWait)) {
                            ok = false;
                            break;
                        }
                        mbar_expect_tx(&fullB[q], (uint32_t)(kAPlanes * bbytes));
                        bulk_g2s(smem + q * stage_bytes + kAPlanes * kABytes, ug + (size_t)ks * kAPlanes * bbytes,
                                 (uint32_t)(kAPlanes * bbytes), &fullB[q]);
                    }
                }
            } else if (warp == 5) {
                if (lane == 0) {  // MMA issuer
                    for (int ks = 0; ks < KS && ok; ks++) {
                        const uint32_t it = it0 + ks, q = it % S, par = (it / S) & 1u;
                        if (!mbar_wait_bounded(&fullA[q], par, kSplitWait) || !mbar_wait_bounded(&fullB[q], par, kSplitWait)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t a = smem_u32(smem + q * stage_bytes);
                        const uint64_t xrh = umma_desc_kmajor(a), xrl = umma_desc_kmajor(a + kABytes);
                        const uint64_t xih = umma_desc_kmajor(a + 2 * kABytes), xil = umma_desc_kmajor(a + 3 * kABytes);
                        const uint32_t b = a + kAPlanes * kABytes;
                        const uint64_t urh = umma_desc_kmajor(b), url = umma_desc_kmajor(b + bbytes);
                        const uint64_t uih = umma_desc_kmajor(b + 2 * bbytes), uil = umma_desc_kmajor(b + 3 * bbytes);
                        const uint32_t acc = ks > 0 ? 1u : 0u;
                        const uint32_t dre = tmem, dim = tmem + (uint32_t)MDs;
                        // Re y += Xr Ur - Xi Ui
                        umma_bf16(dre, xrh, urh, idesc, acc);
                        umma_bf16(dre, xrh, url, idesc, 1u);
                        umma_bf16(dre, xrl, urh, idesc, 1u);
                        umma_bf16(dre, xih, uih, idesc_neg, 1u);
                        umma_bf16(dre, xih, uil, idesc_neg, 1u);
                        umma_bf16(dre, xil, uih, idesc_neg, 1u);
                        // Im y += Xr Ui + Xi Ur
                        umma_bf16(dim, xrh, uih, idesc, acc);
                        umma_bf16(dim, xrh, uil, idesc, 1u);
                        umma_bf16(dim, xrl, uih, idesc, 1u);
                        umma_bf16(dim, xih, urh, idesc, 1u);
                        umma_bf16(dim, xih, url, idesc, 1u);
                        umma_bf16(dim, xil, urh, idesc, 1u);
                        umma_commit(&empty[q]);  // frees the stage once these MMAs have read it
                    }
                    umma_commit(&accf);
                }
            } else {
                // warps 14-15: the tile's state records, loaded while the MMAs run
                for (int m = tid - 448; m < rows; m += 64) load_state(&s_st[m], &P.st[s_tr[m]]);
            }
            // lanes 1-31 of the B-producer and MMA warps park here until their lane 0 is done: spinning on
            // the accumulator barrier instead would take the warp's issue slots from the lane issuing
            __syncwarp();
            kit += (uint32_t)KS;
            if (!ok) atomicExch(&s_fail, 1);
            // accumulator complete (every thread waits on the commit); the ring is free afterwards
            if (!mbar_wait_bounded(&accf, ntile & 1u, kSplitWait)) atomicExch(&s_fail, 1);
            tc_fence_after();
            __syncthreads();
            if (s_fail) {
                ok = false;
                break;
            }
            const long long t2 = clock64();
            float *sacc = reinterpret_cast<float *>(smem);  // [RP][2 MDs + 1] FP32 accumulators
            const int SR = 2 * MDs + 1;
            for (int p0 = 0; p0 < rows; p0 += RP) {  // passes of RP trajectories
                const long long ts = clock64();
                const int q = warp & 3;  // TMEM lanes 32q..32q+31 belong to warps q, q+4, q+8, q+12
                if (32 * q >= p0 && 32 * q < p0 + RP && 32 * q < rows) {
                    const uint32_t lanes = tmem + ((uint32_t)(32 * q) << 16);
                    float *dst = sacc + (size_t)(32 * q - p0 + lane) * SR;
                    for (int r0 = 8 * (warp >> 2); r0 < MDs; r0 += 32) {  // 8 output rows at a time
                        float vr[8], vi[8];
                        tmem_ld8x2(lanes + (uint32_t)r0, lanes + (uint32_t)(MDs + r0), vr, vi);
    #pragma unroll
                        for (int i = 0; i < 8; i++) {
                            dst[r0 + i] = vr[i];
                            dst[MDs + r0 + i] = vi[i];
                        }
                    }
                }
                tc_fence_before();
                __syncthreads();
                tr_stage += clock64() - ts;
                // every warp runs its trajectories (columns warp, warp + 16, ...) through the epilogue,
                // then appends them to their next buckets with one atomic each, all in flight together
                const int pn = min(RP, rows - p0);
                int nm = 0;
                for (int cc = warp; cc < pn; cc += kThreads / 32, nm++) {
                    const int m = p0 + cc;
                    const float *row = sacc + (size_t)cc * SR;
                    for (int k = lane; k < MDs; k += 32) wcol[k] = make_double2((double)row[k], (double)row[MDs + k]);
                    __syncwarp();
                    const int g2 = column_epilogue(P, wcol, s_tr[m], s_st[m], lane);
                    if (lane == 0) w_g2[warp][nm] = g2;
                    __syncwarp();
                }
                if (lane < nm) {
                    const int g2 = w_g2[warp][lane];
                    const int tr = s_tr[p0 + warp + (kThreads / 32) * lane];
                    if (g2 >= 0) {
                        const int pos = atomicAdd(&cnt_next[g2], 1);
                        list_next[P.g_loff[g2] + pos] = tr;
                    } else if (g2 == kRecheck) {
                        rlist_next[atomicAdd(rcnt_next, 1)] = tr;
                    }
                }
                fence_proxy_async();  // generic writes to the ring before the next tile's bulk copies
                __syncthreads();
            }
            work += rows;
            ntile++;
            const long long t3 = clock64();
            tr_setup += t1 - t0;
            tr_mma += t2 - t1;
            tr_epi += t3 - t2;
        }

        steps_done++;
        if (!ok && tid == 0) atomicAdd(&P.ctrl[4], 1);  // every CTA stops after the barrier below
        // the last CTA to finish plans the next micro-step from the buckets all CTAs filled; with a
        // next step in this launch the others wait for that plan (bounded), then read it
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            s_gen = ld_acquire_u32(P.gen);
            s_last = atomicAdd(P.plan_sync, 1u) == gridDim.x - 1;
        }
        __syncthreads();
        const bool more = si + 1 < nsteps;
        if (s_last) {
            __threadfence();
            split_plan(P, cnt_next, __ldcg(rcnt_next), gridDim.x);
            if (tid == 0) {
                *P.plan_sync = 0u;
                __threadfence();
                st_release_u32(P.gen, s_gen + 1u);
            }
        } else if (more && tid == 0) {
            long long i = 0;
            while (ld_acquire_u32(P.gen) == s_gen && i < kGridWait) i++;
            if (i == kGridWait) {
                atomicAdd(&P.ctrl[4], 1);
                report_error(P, -1, ERR_TIMEOUT);
            }
        }
        __syncthreads();
        __threadfence();
        if (!more || !ok || __ldcg(P.ctrl + 4) != 0) break;
    }  // micro-steps

    if (!ok) {
        // give the copies and MMAs still in flight time to land before the memory goes away
        if (warp == 5 && lane == 0) {
            umma_commit(&accf);
            mbar_wait_bounded(&accf, ntile & 1u, kSplitWait);
        }
        if (warp == 4 && lane == 0) {
            for (int q = 0; q < S; q++) {
                mbar_wait_bounded(&fullB[q], 0u, 1024);
                mbar_wait_bounded(&fullB[q], 1u, 1024);
            }
            for (int q = 0; q < 2; q++) {
                mbar_wait_bounded(&rbar[q], 0u, 1024);
                mbar_wait_bounded(&rbar[q], 1u, 1024);
            }
        }
        if (tid == 0) report_error(P, -1, ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols)
                     : "memory");
    }
    if (tid == 0 && work) atomicAdd((unsigned long long *)P.work, (unsigned long long)work);
    if (tid == 0 && ntile) atomicAdd((unsigned long long *)(P.work + 1), (unsigned long long)ntile);
    if (tid == 0 && nrechk) atomicAdd((unsigned long long *)(P.work + 2), (unsigned long long)nrechk);
    if (P.trace && tid == 0) {  // fields: total, setup, -, MMA phase, epilogue, tiles, TMEM staging, rows
        long long *tr = P.trace + (size_t)blockIdx.x * kTraceFields;
        tr[0] += clock64() - t_begin;
        tr[1] += tr_setup;
        tr[3] += tr_mma;
        tr[4] += tr_epi;
        tr[5] += ntile;
        tr[6] += tr_stage;
        tr[7] += work;
    }
    if (blockIdx.x == 0 && tid == 0 && steps_done) atomicAdd(P.sdone, steps_done);
}
