// qjx_tree.cu -- split trees (the QJ propagators U_{b,l} = exp(K_b dt_{b,l})) built on the GPU.
//
// The reference exponentiates every level of every branch on the host (Eigen exp(),
// QJX/qj_proc.cpp:55,98), and so does qjx_build_dimer (Higham's Pade scaling and squaring, one
// level at a time).  At d = 1024 that is about a minute of host time per ensemble, which a
// serving loop cannot spend per request.  Here the levels are related as the tree is: dt halves
// from one level to the next, so U_l = U_{l+1}^2.  The finest level is a Taylor series of the
// scaled generator X = K dt / 2^s with ||X||_1 <= 1/4 (degree 14: remainder below 1e-19 of ||e^X||),
// squared s times; every coarser level is one squaring.  All products are FP64 complex GEMMs in a
// plain shared-memory tiled kernel (setup work, not the hot path).
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "../../include/qjx_b200.h"

namespace tree {

constexpr int BM = 64, BN = 64, BK = 8, TX = 16;  // 256 threads, 4 x 4 complex outputs each

// C = A B for n x n complex row-major matrices.
__global__ void __launch_bounds__(256) zgemm_kernel(int n, const double2 *A, const double2 *B, double2 *C)
{
    __shared__ double2 As[BK][BM];
    __shared__ double2 Bs[BK][BN];
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int row0 = blockIdx.y * BM, col0 = blockIdx.x * BN;
    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0.0, 0.0);
    for (int k0 = 0; k0 < n; k0 += BK) {
        for (int e = tid; e < BM * BK; e += 256) {
            const int m = e / BK, k = e % BK, r = row0 + m, kk = k0 + k;
            As[k][m] = (r < n && kk < n) ? A[(size_t)r * n + kk] : make_double2(0.0, 0.0);
        }
        for (int e = tid; e < BK * BN; e += 256) {
            const int k = e / BN, c = e % BN, kk = k0 + k, cc = col0 + c;
            Bs[k][c] = (kk < n && cc < n) ? B[(size_t)kk * n + cc] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; k++) {
            double2 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[k][ty + TX * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[k][tx + TX * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    double2 &c = acc[i][j];
                    c.x = __fma_rn(a[i].x, b[j].x, c.x);
                    c.x = __fma_rn(-a[i].y, b[j].y, c.x);
                    c.y = __fma_rn(a[i].x, b[j].y, c.y);
                    c.y = __fma_rn(a[i].y, b[j].x, c.y);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int r = row0 + ty + TX * i, c = col0 + tx + TX * j;
            if (r < n && c < n) C[(size_t)r * n + c] = acc[i][j];
        }
}

// T = I + P / k (a Horner step of the Taylor series; P may be T)
__global__ void horner_kernel(int n, const double2 *P, double k, double2 *T)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n) return;
    const double2 p = P[e];
    const bool diag = (e / n) == (e % n);
    T[e] = make_double2(__dadd_rn(diag ? 1.0 : 0.0, __ddiv_rn(p.x, k)), __ddiv_rn(p.y, k));
}

// X = s K (complex K, real s)
__global__ void scale_kernel(int n, const double2 *K, double s, double2 *X)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n) return;
    X[e] = make_double2(__dmul_rn(K[e].x, s), __dmul_rn(K[e].y, s));
}

static cudaError_t gemm(int n, const double2 *A, const double2 *B, double2 *C, cudaStream_t st)
{
    const dim3 grid((n + BN - 1) / BN, (n + BM - 1) / BM);
    zgemm_kernel<<<grid, 256, 0, st>>>(n, A, B, C);
    return cudaGetLastError();
}

}  // namespace tree

extern "C" qjx_status qjx_expm_tree(int d, int nb, const double *K, const double *head, int deep, int device,
                                    double *Utree)
{
    using namespace tree;
    if (d < 1 || nb < 1 || deep < 1 || deep > 62 || !K || !head || !Utree) return QJX_ERR_INVALID_ARG;
    for (int b = 0; b < nb; b++)
        if (!(head[b] > 0.0)) return QJX_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return QJX_ERR_CUDA;
    // a private stream and stream-ordered allocations: no device-wide synchronisation, so trees can
    // be built while engines run on the same device
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return QJX_ERR_CUDA;
    const size_t dd = (size_t)d * d, bytes = dd * sizeof(double2);
    double2 *dK = nullptr, *X = nullptr, *T = nullptr, *P = nullptr;
    qjx_status status = QJX_OK;
    if (cudaMallocAsync(&dK, bytes, st) != cudaSuccess || cudaMallocAsync(&X, bytes, st) != cudaSuccess ||
        cudaMallocAsync(&T, bytes, st) != cudaSuccess || cudaMallocAsync(&P, bytes, st) != cudaSuccess)
        status = QJX_ERR_OOM;
    const int eb = 256, eg = (int)((dd + eb - 1) / eb);
    for (int b = 0; b < nb && status == QJX_OK; b++) {
        const double *Kb = K + 2 * dd * b;
        // the finest level's step and the 1-norm of K dt (largest column sum of |K_ij|), on the host
        const double dt = std::ldexp(head[b], -(deep + 1));
        double norm1 = 0.0;
        for (int j = 0; j < d; j++) {
            double s = 0.0;
            for (int i = 0; i < d; i++) s += std::hypot(Kb[2 * ((size_t)i * d + j)], Kb[2 * ((size_t)i * d + j) + 1]);
            norm1 = std::max(norm1, s);
        }
        norm1 *= dt;
        int sq = 0;
        while (std::ldexp(norm1, -sq) > 0.25) sq++;
        if (cudaMemcpyAsync(dK, Kb, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            status = QJX_ERR_CUDA;
            break;
        }
        scale_kernel<<<eg, eb, 0, st>>>(d, dK, std::ldexp(dt, -sq), X);
        // Horner: T = I; T = I + X T / k for k = 14 .. 1
        cudaMemsetAsync(T, 0, bytes, st);
        horner_kernel<<<eg, eb, 0, st>>>(d, T, 1.0, T);  // T = I
        for (int k = 14; k >= 1; k--) {
            if (gemm(d, X, T, P, st) != cudaSuccess) status = QJX_ERR_CUDA;
            horner_kernel<<<eg, eb, 0, st>>>(d, P, (double)k, T);
        }
        for (int i = 0; i < sq; i++) {  // (e^X)^(2^sq)
            if (gemm(d, T, T, P, st) != cudaSuccess) status = QJX_ERR_CUDA;
            std::swap(T, P);
        }
        // levels deep-1 .. 0: each the square of the next finer one
        for (int l = deep - 1; l >= 0 && status == QJX_OK; l--) {
            if (l < deep - 1) {
                if (gemm(d, T, T, P, st) != cudaSuccess) status = QJX_ERR_CUDA;
                std::swap(T, P);
            }
            if (cudaMemcpyAsync(Utree + 2 * dd * ((size_t)b * deep + l), T, bytes, cudaMemcpyDeviceToHost, st) !=
                cudaSuccess)
                status = QJX_ERR_CUDA;
        }
    }
    cudaFreeAsync(dK, st);
    cudaFreeAsync(X, st);
    cudaFreeAsync(T, st);
    cudaFreeAsync(P, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) status = QJX_ERR_CUDA;
    cudaStreamDestroy(st);
    return status;
}
