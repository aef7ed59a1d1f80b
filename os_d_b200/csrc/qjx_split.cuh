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
// runs unchanged (norm test, jump, renormalisation, observables).
//
// Shared-memory operands use the K-major no-swizzle canonical layout: a core matrix is
// 8 rows x 16 bytes (8 bf16 along K) stored contiguously; within one k-step (16 bf16 of K)
// the two K-halves of a row group are 128 bytes apart (leading byte offset) and consecutive
// 8-row groups 256 bytes apart (stride byte offset).  The host writes B in exactly this
// order, so one k-step of all four B planes is one contiguous TMA bulk copy.
//
// Per tile (one matrix, up to 128 trajectories) a ring of S stages (as many as shared memory
// holds, 5 at d = 201), one k-step of A and B planes each:
//   warps 0-3, 6-9, 10-13   three producer groups, one thread per trajectory row; group p
//               converts the k-steps ks = p (mod 3): FP64 state -> bf16 planes of A (generic
//               stores, then fence.proxy.async and an arrive on fullA)
//   warp 4      one thread issues the bulk copy of the B planes (complete_tx on fullB)
//   warp 5      one thread issues the 12 tcgen05.mma of a k-step and commits them to empty[stage]
// then the accumulators (commit to accf) are read by the warps whose TMEM lane quarter holds
// each group of 32 trajectories, staged as FP64 columns in the (now idle) ring, and run
// through column_epilogue.  Rows per tile are chosen per micro-step so that the tiles fit
// one wave of CTAs.

constexpr int kAPlanes = 4;                  // A and B planes: Re hi, Re lo, Im hi, Im lo
constexpr int kTileM = 128;                  // MMA M = TMEM lanes (a tile holds up to 128 trajectories)
constexpr int kMaxSStages = 8;               // operand ring depth (runtime: as deep as shared memory allows)
constexpr int kABytes = kTileM * 32;         // one plane of one k-step of A: 128 rows x 16 bf16
constexpr int kTmemCols = 512;
constexpr long long kSplitWait = 1ll << 20;  // bounded mbarrier polls (normal waits end within microseconds)

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

// 8 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v)
{
    uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
                 : "r"(taddr));
    // the registers are valid after wait::ld; tying them to the wait keeps every use behind it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7)
                 :
                 : "memory");
    v[0] = __uint_as_float(r0);
    v[1] = __uint_as_float(r1);
    v[2] = __uint_as_float(r2);
    v[3] = __uint_as_float(r3);
    v[4] = __uint_as_float(r4);
    v[5] = __uint_as_float(r5);
    v[6] = __uint_as_float(r6);
    v[7] = __uint_as_float(r7);
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

// Dynamic shared memory: a ring of `stages` operand stages, each [A planes][B planes] of one
// k-step; after the MMAs of a tile the ring holds the FP64 epilogue columns (32 x (MDs+1)),
// the per-warp epilogue scratch (16 x MD) and the tile's 128 trajectory records.
size_t split_stage_bytes(int MDs) { return (size_t)kAPlanes * (kABytes + (size_t)MDs * 32); }

size_t split_smem_bytes(int MDs, int MD, int stages)
{
    const size_t ring = (size_t)stages * split_stage_bytes(MDs);
    (void)MD;
    const size_t epi = (size_t)32 * (MDs + 1) * sizeof(double2) + (size_t)kTileM * sizeof(TrajState);
    return ring > epi ? ring : epi;
}

__global__ void __launch_bounds__(kThreads, 1) split_step_kernel(const Params P, int s)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int MDs = P.MDs, KS = P.KS, S = P.sstages;
    const int bbytes = MDs * 32;                               // one plane of one k-step of B
    const size_t stage_bytes = (size_t)kAPlanes * (kABytes + bbytes);
    const int S16 = MDs + 1;
    double2 *Bt = reinterpret_cast<double2 *>(smem);          // epilogue: [32][S16] FP64 columns
    TrajState *s_st = reinterpret_cast<TrajState *>(Bt + 32 * S16);  // [128]
    __shared__ __align__(8) uint64_t fullA[kMaxSStages], fullB[kMaxSStages], empty[kMaxSStages], accf;
    __shared__ uint32_t s_tmem;
    __shared__ int s_tstart[kMaxGroups + 1];
    __shared__ int s_tr[kTileM];
    __shared__ long long s_src[kTileM];
    __shared__ int s_fail;
    __shared__ int s_rows;  // trajectories per tile in this micro-step
    __shared__ int cnt_cur[kMaxGroups];  // bucket sizes of this step, read once in parallel
    __shared__ int s_g2[kTileM];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = P.G, n = P.n, d = P.d;
    int *cnt_next = P.cnt + ((s + 1) % 3) * G;
    const int *list_cur = P.lists + (size_t)(s & 1) * P.ltot;
    int *list_next = P.lists + (size_t)((s + 1) & 1) * P.ltot;

    for (int i = tid; i < G; i += kThreads) cnt_cur[i] = P.cnt[(s % 3) * G + i];
    if (blockIdx.x == 0)
        for (int i = tid; i < G; i += kThreads) P.cnt[((s + 2) % 3) * G + i] = 0;
    __syncthreads();
    if (warp == 0) {
        // rows per tile: the smallest multiple of 8 (<= 128) whose tiles fit one wave of CTAs, so
        // the trajectories (and their epilogues) spread over all SMs; 128 when none does
        int tiles = 0;
        if (lane < 16)
            for (int g = 0; g < G; g++) tiles += (cnt_cur[g] + 8 * lane + 7) / (8 * lane + 8);
        const unsigned fit = __ballot_sync(0xffffffffu, lane < 16 && tiles <= (int)gridDim.x);
        const int R = fit ? 8 * (__ffs(fit)) : kTileM;
        if (lane == 0) {
            s_rows = R;
            int acc = 0;
            for (int g = 0; g < G; g++) {
                s_tstart[g] = acc;
                acc += (cnt_cur[g] + R - 1) / R;
            }
            s_tstart[G] = acc;
            for (int q = 0; q < S; q++) {
                mbar_init(&fullA[q], kTileM);
                mbar_init(&fullB[q], 1);
                mbar_init(&empty[q], 1);
            }
            mbar_init(&accf, 1);
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
    const int T = s_tstart[G];
    const uint32_t idesc = umma_idesc_bf16(kTileM, MDs);
    const uint32_t idesc_neg = idesc | (1u << 13);  // negate A
    long long work = 0;
    uint32_t ntile = 0;
    bool ok = true;
    long long tr_setup = 0, tr_mma = 0, tr_stage = 0, tr_epi = 0;
    const long long t_begin = clock64();

    for (int t = blockIdx.x; t < T && ok; t += gridDim.x, ntile++) {
        const long long t0 = clock64();
        int lo = 0, hi = G;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_tstart[mid] <= t) lo = mid;
            else hi = mid;
        }
        const int g = lo;
        const int base = (t - s_tstart[g]) * s_rows;
        const int rows = min(s_rows, cnt_cur[g] - base);
        if (tid < kTileM) {
            if (tid < rows) {
                const int tr = list_cur[P.g_loff[g] + base + tid];
                const int slot = src_slot(P.st[tr].phase, P.st[tr].cur, P.st[tr].rk_stage);
                s_tr[tid] = tr;
                s_src[tid] = ((long long)slot * n + tr) * P.MD;
            } else {
                s_tr[tid] = -1;
                s_src[tid] = -1;
            }
        }
        __syncthreads();
        const long long t1 = clock64();
        const uint32_t it0 = ntile * (uint32_t)KS;  // k-steps issued before this tile

        const int agrp = (warp < 4) ? 0 : (warp >= 6 && warp < 10) ? 1 : (warp >= 10 && warp < 14) ? 2 : -1;
        if (agrp >= 0) {
            // A producers: group p (4 warps, thread m = row m) handles the k-steps ks = p (mod 3), so
            // three independent load-convert chains run in parallel; each thread issues its loads
            // before waiting for the stage to drain
            const int m = tid - (agrp == 0 ? 0 : (agrp == 1 ? 192 : 320));
            const double2 *src = (s_src[m] >= 0) ? P.psi + s_src[m] : nullptr;
            const int off = (m & 7) * 16 + (m >> 3) * 256;
            for (int ks = agrp; ks < KS && ok; ks += 3) {
                const uint32_t it = it0 + ks, q = it % S;
                unsigned char *As = smem + q * stage_bytes + off;
                for (int hh = 0; hh < 2; hh++) {  // K-halves: components 16 ks + 8 hh .. + 7
                    double2 v[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const int k = 16 * ks + 8 * hh + i;
                        v[i] = (src && k < d) ? src[k] : make_double2(0.0, 0.0);
                    }
                    if (hh == 0 && it >= (uint32_t)S && !mbar_wait_bounded(&empty[q], ((it / S) - 1) & 1u, kSplitWait))
                        ok = false;
                    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        split_pair(make_double2(v[2 * j].x, v[2 * j + 1].x), rh[j], rl[j]);
                        split_pair(make_double2(v[2 * j].y, v[2 * j + 1].y), ih[j], il[j]);
                    }
                    *reinterpret_cast<uint4 *>(As + 128 * hh) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
                    *reinterpret_cast<uint4 *>(As + kABytes + 128 * hh) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
                    *reinterpret_cast<uint4 *>(As + 2 * kABytes + 128 * hh) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
                    *reinterpret_cast<uint4 *>(As + 3 * kABytes + 128 * hh) = make_uint4(il[0], il[1], il[2], il[3]);
                }
                fence_proxy_async();
                mbar_arrive(&fullA[q]);
            }
        } else if (warp == 4) {
            if (lane == 0) {  // B producer
                const unsigned char *ug = P.usplit + (size_t)g * KS * kAPlanes * bbytes;
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
        }
        if (!ok) atomicExch(&s_fail, 1);
        // accumulator complete (every thread waits on the commit); the ring is free afterwards
        if (!mbar_wait_bounded(&accf, ntile & 1u, kSplitWait)) atomicExch(&s_fail, 1);
        tc_fence_after();
        __syncthreads();
        if (s_fail) {
            ok = false;
            break;
        }
        // the tile's state records, all loaded at once (one L2 round trip for the whole tile)
        for (int m = tid; m < rows; m += kThreads) load_state(&s_st[m], &P.st[s_tr[m]]);
        const long long t2 = clock64();
        for (int c = 0; c < 4 && 32 * c < rows; c++) {
            const long long ts = clock64();
            if ((warp & 3) == c) {  // TMEM lanes 32c..32c+31 belong to warps c, c+4, c+8, c+12
                const uint32_t lanes = tmem + ((uint32_t)(32 * c) << 16);
                for (int r0 = 8 * (warp >> 2); r0 < MDs; r0 += 32) {  // 8 output rows at a time
                    float vr[8], vi[8];
                    tmem_ld8(lanes + (uint32_t)r0, vr);
                    tmem_ld8(lanes + (uint32_t)(MDs + r0), vi);
                    double2 *dst = Bt + (size_t)lane * S16 + r0;
#pragma unroll
                    for (int i = 0; i < 8; i++) dst[i] = make_double2((double)vr[i], (double)vi[i]);
                }
            }
            tc_fence_before();
            __syncthreads();
            tr_stage += clock64() - ts;
            for (int cc = warp; cc < 32; cc += kThreads / 32) {
                const int m = 32 * c + cc;
                if (m < rows) {
                    const int g2 = column_epilogue(P, Bt + (size_t)cc * S16, s_tr[m], s_st[m], lane);
                    if (lane == 0) s_g2[m] = g2;
                }
            }
            fence_proxy_async();  // generic writes to the ring before the next tile's bulk copies
            __syncthreads();
        }
        __syncthreads();
        enqueue_batch(P, cnt_next, list_next, s_tr, s_g2, rows);
        work += rows;
        const long long t3 = clock64();
        tr_setup += t1 - t0;
        tr_mma += t2 - t1;
        tr_epi += t3 - t2;
    }

    if (!ok) {
        // give the copies and MMAs still in flight time to land before the memory goes away
        if (warp == 5 && lane == 0) {
            umma_commit(&accf);
            mbar_wait_bounded(&accf, ntile & 1u, kSplitWait);
        }
        if (warp == 4 && lane == 0)
            for (int q = 0; q < S; q++) {
                mbar_wait_bounded(&fullB[q], 0u, 1024);
                mbar_wait_bounded(&fullB[q], 1u, 1024);
            }
        if (tid == 0) {
            atomicAdd(&P.ctrl[4], 1);
            report_error(P, -1, ERR_TIMEOUT);
        }
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
}
