// qjx_split.cuh -- the split-precision micro-step on the tcgen05 tensor cores (precision 1).
//
// Same lock-step micro-steps, buckets and trajectory state machine as the FP64 plain form;
// only the d x d complex matvec changes.  Roles are transposed against the FP64 kernel so that
// the trajectory, not the matrix row, is the MMA M dimension:
//
//   D[m][n] = sum_kk A[m][kk] B[n][kk]      m: trajectory of the tile (128 = TMEM lanes)
//                                           n: 2 r + {0, 1}  (Re, Im of output row r)
//                                          kk: 2 k + {0, 1}  (Re, Im of input component k)
//   A = the tile's states as bf16 planes (written by the CTA from the FP64 states),
//   B = the real block form [[Re M, -Im M], [Im M, Re M]] of the bucket's matrix, rows and
//       columns interleaved, as bf16 planes prepared once by the host,
//   D = FP32 accumulator in tensor memory, 2 MDs columns (two MMA N-halves of MDs each).
//
// Every operand x is split x = hi + lo with hi = bf16(x), lo = bf16(x - hi); the MMAs add
// hi*hi + hi*lo + lo*hi in FP32 ("bf16x3"), which leaves about 2^-16 of relative error per
// product and the FP32 accumulation error (measured about 4e-6 of max|y| per matvec at
// d = 201).  The accumulator is read back to FP64 and the FP64 epilogue of the plain form runs
// unchanged (norm test, jump, renormalisation, observables).
//
// Shared-memory operands use the K-major no-swizzle canonical layout: a core matrix is
// 8 rows x 16 bytes (8 bf16 along K) stored contiguously; within one k-step (16 bf16 of K)
// the two K-halves of a row group are 128 bytes apart (leading byte offset) and consecutive
// 8-row groups 256 bytes apart (stride byte offset).  The host writes B in exactly this
// order, so one k-step of all planes is one contiguous TMA bulk copy.
//
// Per tile (one matrix, up to 128 trajectories) and k-step, a 3-stage ring:
//   warps 0-3   one thread per trajectory row: FP64 state -> bf16 planes of A (generic
//               stores, then fence.proxy.async and an arrive on fullA)
//   warp 4      one thread issues the bulk copy of the B planes (complete_tx on fullB)
//   warp 5      one thread issues the 2 x 3 tcgen05.mma and commits them to empty[stage]
// then the accumulator (commit to accf) is read by the warps whose TMEM lane quarter holds
// each group of 32 trajectories, staged as FP64 columns, and run through column_epilogue.

constexpr int kPlanes = 2;                   // bf16 hi, lo
constexpr int kTileM = 128;                  // trajectories per tile (TMEM lanes, MMA M)
constexpr int kSStages = 3;                  // operand ring depth
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

// bf16 round-to-nearest-even of a double (through the exact FP32 value when it is exact,
// else rounding the double once to bf16 precision); returns the 16-bit pattern.
__device__ __forceinline__ uint32_t bf16_bits(double x)
{
    return (uint32_t)__bfloat16_as_ushort(__double2bfloat16(x));
}

__device__ __forceinline__ double bf16_value(uint32_t b)
{
    return (double)__uint_as_float(b << 16);
}

// hi/lo planes of one (re, im) pair packed as two bf16 (re in the low half: lower address).
__device__ __forceinline__ void split_pair(double2 v, uint32_t &hi, uint32_t &lo)
{
    const uint32_t hr = bf16_bits(v.x), hm = bf16_bits(v.y);
    const uint32_t lr = bf16_bits(v.x - bf16_value(hr)), lm = bf16_bits(v.y - bf16_value(hm));
    hi = hr | (hm << 16);
    lo = lr | (lm << 16);
}

size_t split_smem_bytes(int MDs)
{
    const size_t bbytes = (size_t)2 * MDs * 32;
    return (size_t)kSStages * kPlanes * (kABytes + bbytes) + (size_t)32 * (MDs + 1) * sizeof(double2);
}

__global__ void __launch_bounds__(kThreads, 1) split_step_kernel(const Params P, int s)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int MDs = P.MDs, KS = P.KS, NP = 2 * MDs;
    const int bbytes = NP * 32;  // one plane of one k-step of B
    unsigned char *As = smem;                                          // [stage][plane][kABytes]
    unsigned char *Bs = As + kSStages * kPlanes * kABytes;            // [stage][plane][bbytes]
    const int S16 = MDs + 1;
    double2 *Bt = reinterpret_cast<double2 *>(Bs + (size_t)kSStages * kPlanes * bbytes);  // [32][S16]
    __shared__ __align__(8) uint64_t fullA[kSStages], fullB[kSStages], empty[kSStages], accf;
    __shared__ uint32_t s_tmem;
    __shared__ int s_tstart[kMaxGroups + 1];
    __shared__ int s_tr[kTileM];
    __shared__ long long s_src[kTileM];
    __shared__ int s_fail;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = P.G, n = P.n, d = P.d;
    const int *cnt_cur = P.cnt + (s % 3) * G;
    int *cnt_next = P.cnt + ((s + 1) % 3) * G;
    const int *list_cur = P.lists + (size_t)(s & 1) * G * n;
    int *list_next = P.lists + (size_t)((s + 1) & 1) * G * n;

    if (blockIdx.x == 0)
        for (int i = tid; i < G; i += kThreads) P.cnt[((s + 2) % 3) * G + i] = 0;
    if (tid == 0) {
        int acc = 0;
        for (int g = 0; g < G; g++) {
            s_tstart[g] = acc;
            acc += (cnt_cur[g] + kTileM - 1) / kTileM;
        }
        s_tstart[G] = acc;
        for (int q = 0; q < kSStages; q++) {
            mbar_init(&fullA[q], kTileM);
            mbar_init(&fullB[q], 1);
            mbar_init(&empty[q], 1);
        }
        mbar_init(&accf, 1);
        s_fail = 0;
        fence_proxy_async();
    }
    if (warp == 0) {  // the whole tensor memory of the SM (one CTA per SM)
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
    long long work = 0;
    uint32_t ntile = 0;
    bool ok = true;

    for (int t = blockIdx.x; t < T && ok; t += gridDim.x, ntile++) {
        int lo = 0, hi = G;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_tstart[mid] <= t) lo = mid;
            else hi = mid;
        }
        const int g = lo;
        const int base = (t - s_tstart[g]) * kTileM;
        const int rows = min(kTileM, cnt_cur[g] - base);
        if (tid < kTileM) {
            if (tid < rows) {
                const int tr = list_cur[(size_t)g * n + base + tid];
                const int ph = P.st[tr].phase, cur = P.st[tr].cur;
                const int slot = (ph >= PH_OBS_E) ? (cur ^ 1) : cur;
                s_tr[tid] = tr;
                s_src[tid] = ((long long)slot * n + tr) * P.MD;
            } else {
                s_tr[tid] = -1;
                s_src[tid] = -1;
            }
        }
        __syncthreads();
        const uint32_t it0 = ntile * (uint32_t)KS;  // k-steps issued before this tile

        if (warp < 4) {
            // A producer: thread m writes row m of every k-step
            const int m = tid;
            const double2 *src = (s_src[m] >= 0) ? P.psi + s_src[m] : nullptr;
            const int off = (m & 7) * 16 + (m >> 3) * 256;
            for (int ks = 0; ks < KS && ok; ks++) {
                const uint32_t it = it0 + ks, q = it % kSStages;
                if (it >= kSStages && !mbar_wait_bounded(&empty[q], ((it / kSStages) - 1) & 1u, kSplitWait)) ok = false;
                uint32_t h[8], l[8];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int k = 8 * ks + i;
                    const double2 v = (src && k < d) ? src[k] : make_double2(0.0, 0.0);
                    split_pair(v, h[i], l[i]);
                }
                uint4 *ah = reinterpret_cast<uint4 *>(As + (q * kPlanes + 0) * kABytes + off);
                uint4 *al = reinterpret_cast<uint4 *>(As + (q * kPlanes + 1) * kABytes + off);
                ah[0] = make_uint4(h[0], h[1], h[2], h[3]);
                ah[8] = make_uint4(h[4], h[5], h[6], h[7]);  // +128 bytes: second K-half
                al[0] = make_uint4(l[0], l[1], l[2], l[3]);
                al[8] = make_uint4(l[4], l[5], l[6], l[7]);
                fence_proxy_async();
                mbar_arrive(&fullA[q]);
            }
        } else if (warp == 4) {
            if (lane == 0) {  // B producer
                const unsigned char *ug = P.usplit + (size_t)g * KS * kPlanes * bbytes;
                for (int ks = 0; ks < KS && ok; ks++) {
                    const uint32_t it = it0 + ks, q = it % kSStages;
                    if (it >= kSStages && !mbar_wait_bounded(&empty[q], ((it / kSStages) - 1) & 1u, kSplitWait)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&fullB[q], (uint32_t)(kPlanes * bbytes));
                    bulk_g2s(Bs + (size_t)q * kPlanes * bbytes, ug + (size_t)ks * kPlanes * bbytes,
                             (uint32_t)(kPlanes * bbytes), &fullB[q]);
                }
            }
        } else if (warp == 5) {
            if (lane == 0) {  // MMA issuer
                for (int ks = 0; ks < KS && ok; ks++) {
                    const uint32_t it = it0 + ks, q = it % kSStages, par = (it / kSStages) & 1u;
                    if (!mbar_wait_bounded(&fullA[q], par, kSplitWait) || !mbar_wait_bounded(&fullB[q], par, kSplitWait)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(As + (q * kPlanes + 0) * kABytes);
                    const uint32_t a1 = smem_u32(As + (q * kPlanes + 1) * kABytes);
                    const uint32_t b0 = smem_u32(Bs + (size_t)(q * kPlanes + 0) * bbytes);
                    const uint32_t b1 = smem_u32(Bs + (size_t)(q * kPlanes + 1) * bbytes);
#pragma unroll
                    for (int hn = 0; hn < 2; hn++) {
                        const uint32_t bo = (uint32_t)hn * (uint32_t)(MDs / 8) * 256u;  // N-half: MDs rows
                        const uint32_t dcol = tmem + (uint32_t)(hn * MDs);
                        umma_bf16(dcol, umma_desc_kmajor(a0), umma_desc_kmajor(b0 + bo), idesc, ks > 0 ? 1u : 0u);
                        umma_bf16(dcol, umma_desc_kmajor(a0), umma_desc_kmajor(b1 + bo), idesc, 1u);
                        umma_bf16(dcol, umma_desc_kmajor(a1), umma_desc_kmajor(b0 + bo), idesc, 1u);
                    }
                    umma_commit(&empty[q]);  // frees the stage once these MMAs have read it
                }
                umma_commit(&accf);
            }
        }
        if (!ok) atomicExch(&s_fail, 1);
        // accumulator complete (every thread waits on the commit)
        if (!mbar_wait_bounded(&accf, ntile & 1u, kSplitWait)) atomicExch(&s_fail, 1);
        tc_fence_after();
        __syncthreads();
        if (s_fail) {
            ok = false;
            break;
        }
        double2 *wscr = reinterpret_cast<double2 *>(Bs) + (size_t)warp * P.MD;  // B ring is free now
        for (int c = 0; c < 4 && 32 * c < rows; c++) {
            if ((warp & 3) == c) {  // TMEM lanes 32c..32c+31 belong to warps c, c+4, c+8, c+12
                const int part = warp >> 2, ncol = NP / 4;
                for (int col = part * ncol; col < (part + 1) * ncol; col += 8) {
                    float v[8];
                    tmem_ld8(tmem + ((uint32_t)(32 * c) << 16) + (uint32_t)col, v);
                    double2 *dst = Bt + (size_t)lane * S16 + col / 2;
#pragma unroll
                    for (int i = 0; i < 4; i++) dst[i] = make_double2((double)v[2 * i], (double)v[2 * i + 1]);
                }
            }
            tc_fence_before();
            __syncthreads();
            for (int cc = warp; cc < 32; cc += kThreads / 32) {
                const int m = 32 * c + cc;
                if (m < rows) column_epilogue(P, Bt + (size_t)cc * S16, wscr, s_tr[m], cnt_next, list_next, lane);
            }
            fence_proxy_async();
            __syncthreads();
        }
        work += rows;
    }

    if (!ok) {
        // give the copies and MMAs still in flight time to land before the memory goes away
        if (warp == 5 && lane == 0) {
            umma_commit(&accf);
            mbar_wait_bounded(&accf, ntile & 1u, kSplitWait);
        }
        if (warp == 4 && lane == 0)
            for (int q = 0; q < kSStages; q++) {
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
}
