// The steps either side of the eigensolve on sm_100a:
//   BS_ORTH   (src/bsr/BSR_MAT3/bs_orth.f90:2-92): orthogonality conditions of
//             the channels imposed on the assembled blocks;
//   rsol_out  (src/bsr/BSR_HD3/rsol_out.f90:20-36): solutions in the B-spline
//             basis and the surface amplitudes WMAT.
//
// BS_ORTH applies, channel after channel, (1 - B zz_i) on the left of the
// blocks in channel row i and (1 - zz_j B) on the right of those in channel
// column j (zz_i = sum of p p^T over the orbitals listed for channel i, B the
// full B-spline overlap).  Matrix products associate, so the result is
// H_ij -> M_i H_ij M_j^T with M_i = 1 - B zz_i for every block at once: two
// batched DGEMMs over the blocks that have a condition on either side.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "ctx.h"

namespace bsrg {
namespace {

// full symmetric overlap from the lower band (Full_mat_sym(ns,ks,sb,bb,'l'), full_mat.f90:2-45)
__global__ void full_from_band_kernel(int ns, int ks, const double *__restrict__ sb, double *__restrict__ B)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= (size_t)ns * ns) return;
    const int i = (int)(q % ns), j = (int)(q / ns);
    const int lo = i > j ? i : j, hi = i > j ? j : i;   // lower-band element (lo, hi)
    const int jp = hi - lo + ks - 1;                     // 0-based band column
    B[q] = (jp >= 0) ? sb[lo + (size_t)ns * jp] : 0.0;
}

__global__ void set_identity_kernel(int ns, int nmat, double *M)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t nn = (size_t)ns * ns;
    if (q >= nn * nmat) return;
    const size_t e = q % nn;
    M[q] = (e % ns == e / ns) ? 1.0 : 0.0;
}

__global__ void gather_columns_kernel(int ns, const double *__restrict__ P, const int *__restrict__ idx, int nidx,
                                      double *__restrict__ out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ns * nidx) return;
    out[q] = P[(q % ns) + (size_t)ns * idx[q / ns]];
}

// WMAT(ich, is) = sum_q bb_ich(ns-1, q) a(ipsol(ich)+q, is): one block per solution, one warp per channel
__global__ void surface_amplitude_kernel(int ns, int nch, const int *__restrict__ ipsol, const double *__restrict__ bb,
                                         int khm, const double *__restrict__ a, double *__restrict__ wmat)
{
    const int is = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int ich = warp; ich < nch; ich += nw) {
        const int j0 = ipsol[ich], m = ipsol[ich + 1] - j0;
        const double *brow = bb + (size_t)ich * ns * ns + (ns - 1);
        double s = 0.0;
        for (int q = lane; q < m; q += 32) s += brow[(size_t)ns * q] * a[(size_t)(j0 + q) + (size_t)khm * is];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) wmat[ich + (size_t)nch * is] = s;
    }
}

__global__ void last_rows_kernel(int ns, int nch, int khm, const double *__restrict__ v, double *__restrict__ wmat)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= (size_t)nch * khm) return;
    const int ich = (int)(q % nch);
    const size_t is = q / nch;
    wmat[q] = v[(size_t)ich * ns + ns - 1 + (size_t)nch * ns * is];
}

// W_OUT (w_out.f90:58-76): per solution is, channel weights WT(ich) = sum over the
// channel's rows j of a(j,is)^2, summed in row order as Fortran's SUM does; then
// SORTA's exchange sort (sorting_routines.f90:79-97) of |WT| gives iprm, and isol is
// the channel of largest weight.  One block per solution; the column passes through
// shared memory in chunks so that the loads are coalesced while each channel's sum
// keeps its sequential order.
constexpr int CW_CHUNK = 2048;

__global__ void channel_weights_kernel(int nch, const int *__restrict__ ipsol, int khm, const double *__restrict__ a,
                                       double *__restrict__ wt, int *__restrict__ isol, int *__restrict__ iprm)
{
    extern __shared__ double cw_sm[];
    double *col = cw_sm;                       // CW_CHUNK
    double *w = col + CW_CHUNK;                // nch
    int *ipt = (int *)(w + nch);               // nch
    const int is = blockIdx.x;
    const double *acol = a + (size_t)khm * is;
    for (int i = threadIdx.x; i < nch; i += blockDim.x) w[i] = 0.0;
    for (int c0 = 0; c0 < khm; c0 += CW_CHUNK) {
        const int c1 = min(c0 + CW_CHUNK, khm);
        __syncthreads();
        for (int j = c0 + threadIdx.x; j < c1; j += blockDim.x) col[j - c0] = acol[j];
        __syncthreads();
        for (int i = threadIdx.x; i < nch; i += blockDim.x) {
            const int j1 = max(ipsol[i], c0), j2 = min(ipsol[i + 1], c1);
            double sum = w[i];
            for (int j = j1; j < j2; j++) sum = __dadd_rn(sum, __dmul_rn(col[j - c0], col[j - c0]));
            w[i] = sum;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nch; i += blockDim.x) wt[i + (size_t)nch * is] = w[i];
    if (threadIdx.x == 0) {
        for (int i = 0; i < nch; i++) ipt[i] = i;
        for (int i1 = 0; i1 < nch - 1; i1++) {
            int j1 = ipt[i1];
            for (int i2 = i1 + 1; i2 < nch; i2++) {
                const int j2 = ipt[i2];
                if (fabs(w[j1]) < fabs(w[j2])) {
                    ipt[i2] = j1;
                    j1 = j2;
                }
            }
            ipt[i1] = j1;
        }
        isol[is] = ipt[0] + 1;
    }
    if (iprm) {
        __syncthreads();
        for (int i = threadIdx.x; i < nch; i += blockDim.x) iprm[i + (size_t)nch * is] = ipt[i] + 1;
    }
}

}  // namespace
}  // namespace bsrg

extern "C" int bsrg_channel_weights(bsrg_ctx *c, int nch, const int *ipsol, int khm, const double *a, double *wt,
                                    int *isol, int *iprm)
{
    using namespace bsrg;
    if (!c || !ipsol || !a || !wt || !isol || nch < 1 || khm < 1 || ipsol[0] != 0 || ipsol[nch] != khm) {
        set_error("bsrg_channel_weights: bad arguments");
        return BSRG_ERR_ARG;
    }
    for (int i = 0; i < nch; i++)
        if (ipsol[i + 1] < ipsol[i]) {
            set_error("bsrg_channel_weights: ipsol decreases at channel %d", i + 1);
            return BSRG_ERR_ARG;
        }
    const size_t shm = sizeof(double) * (CW_CHUNK + (size_t)nch) + sizeof(int) * (size_t)nch;
    int dev_max = 0;
    cudaSetDevice(c->device);
    cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (shm > (size_t)dev_max) {
        set_error("bsrg_channel_weights: nch=%d needs %zu B of shared memory (limit %d)", nch, shm, dev_max);
        return BSRG_ERR_ARG;
    }
    cudaStream_t s = c->stream;
    cudaError_t e;
    int rc = ctx_reserve(c, sizeof(int) * (nch + 1) + 256);
    if (rc != BSRG_OK) return rc;
    if ((rc = ctx_reserve_pinned(c, sizeof(int) * (nch + 1))) != BSRG_OK) return rc;
    if ((e = cudaEventSynchronize(c->ev_stage)) != cudaSuccess) return cuda_fail(e, "channel_weights staging");
    std::memcpy(c->pinned, ipsol, sizeof(int) * (nch + 1));
    int *d_ip = (int *)c->ws;
    if ((e = cudaMemcpyAsync(d_ip, c->pinned, sizeof(int) * (nch + 1), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(e, "channel_weights upload");
    cudaEventRecord(c->ev_stage, s);
    if (shm > 48 * 1024 &&
        (e = smem_attr(channel_weights_kernel, (int)shm)) !=
            cudaSuccess)
        return cuda_fail(e, "channel_weights smem");
    channel_weights_kernel<<<khm, 128, shm, s>>>(nch, d_ip, khm, a, wt, isol, iprm);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "channel_weights");
    return BSRG_OK;
}

extern "C" int bsrg_bs_orth(bsrg_ctx *c, const bsrg_basis *b, int nch, int norb, const double *P, const int *ort_ptr,
                            const int *ort_idx, double *hcc)
{
    using namespace bsrg;
    if (!c || !b || !P || !ort_ptr || !hcc || nch < 1 || norb < 1 || ort_ptr[0] != 0) {
        set_error("bsrg_bs_orth: bad arguments");
        return BSRG_ERR_ARG;
    }
    for (int i = 0; i < nch; i++)
        if (ort_ptr[i + 1] < ort_ptr[i]) {
            set_error("bsrg_bs_orth: ort_ptr must be non-decreasing");
            return BSRG_ERR_ARG;
        }
    const int ntot = ort_ptr[nch];
    for (int q = 0; q < ntot; q++)
        if (!ort_idx || ort_idx[q] < 0 || ort_idx[q] >= norb) {
            set_error("bsrg_bs_orth: orbital index %d out of range (norb %d)", ort_idx ? ort_idx[q] : -1, norb);
            return BSRG_ERR_ARG;
        }
    if (ntot == 0) return BSRG_OK;
    cudaSetDevice(c->device);
    const int ns = b->ns, ks = b->ks;
    const size_t nn = (size_t)ns * ns;
    std::vector<char> has(nch, 0);
    int nmax = 0;
    for (int i = 0; i < nch; i++) {
        has[i] = ort_ptr[i + 1] > ort_ptr[i];
        nmax = ort_ptr[i + 1] - ort_ptr[i] > nmax ? ort_ptr[i + 1] - ort_ptr[i] : nmax;
    }
    // blocks touched: channel row or column with a condition
    std::vector<int> bi, bj;
    for (int i = 0; i < nch; i++)
        for (int j = 0; j <= i; j++)
            if (has[i] || has[j]) {
                bi.push_back(i);
                bj.push_back(j);
            }
    const int nb = (int)bi.size();
    const int chunk = nb < 256 ? nb : 256;
    size_t need = 0;
    auto add = [&](size_t bytes) { need += (bytes + 255) & ~(size_t)255; };
    add(sizeof(double) * nn);                 // B
    add(sizeof(double) * nn * nch);           // M
    add(sizeof(double) * nn);                 // zz
    add(sizeof(double) * ns * nmax);          // selected orbitals
    add(sizeof(int) * ntot);                  // indices
    add(sizeof(double) * nn * chunk);         // T
    add(sizeof(double *) * 3 * chunk * 2);    // pointer arrays (two GEMMs)
    int rc = ctx_reserve(c, need + 256);
    if (rc != BSRG_OK) return rc;
    const size_t pin_bytes = sizeof(int) * ntot + sizeof(double *) * 6 * (size_t)nb + 64;
    if ((rc = ctx_reserve_pinned(c, pin_bytes)) != BSRG_OK) return rc;
    Arena ar{(char *)c->ws, 0, c->ws_bytes};
    double *B = ar.take<double>(nn), *M = ar.take<double>(nn * nch), *zz = ar.take<double>(nn);
    double *Ps = ar.take<double>((size_t)ns * nmax);
    int *d_idx = ar.take<int>(ntot);
    double *T = ar.take<double>(nn * chunk);
    double **d_ptr = ar.take<double *>((size_t)6 * chunk);
    cudaStream_t s = c->stream;
    cudaError_t e;
    // the pinned buffer may still feed an earlier copy on this stream
    if ((e = cudaEventSynchronize(c->ev_stage)) != cudaSuccess) return cuda_fail(e, "bs_orth staging");
    int *h_idx = (int *)c->pinned;
    std::memcpy(h_idx, ort_idx, sizeof(int) * ntot);
    double **h_ptr = (double **)((char *)c->pinned + ((sizeof(int) * ntot + 15) & ~(size_t)15));
    if ((e = cudaMemcpyAsync(d_idx, h_idx, sizeof(int) * ntot, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(e, "bs_orth index upload");
    full_from_band_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(ns, ks, b->sb, B);
    set_identity_kernel<<<(unsigned)((nn * nch + 255) / 256), 256, 0, s>>>(ns, nch, M);
    const double one = 1.0, zero = 0.0, mone = -1.0;
    for (int i = 0; i < nch; i++) {
        if (!has[i]) continue;
        const int nort = ort_ptr[i + 1] - ort_ptr[i];
        gather_columns_kernel<<<(ns * nort + 127) / 128, 128, 0, s>>>(ns, P, d_idx + ort_ptr[i], nort, Ps);
        // zz = Ps Ps^T; M_i = 1 - B zz
        cublasStatus_t b1 = cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, ns, ns, nort, &one, Ps, ns, Ps, ns, &zero,
                                        zz, ns);
        cublasStatus_t b2 = cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, ns, ns, ns, &mone, B, ns, zz, ns, &one,
                                        M + nn * i, ns);
        if (b1 != CUBLAS_STATUS_SUCCESS || b2 != CUBLAS_STATUS_SUCCESS) {
            set_error("bsrg_bs_orth: projector GEMM failed (%d, %d)", (int)b1, (int)b2);
            return BSRG_ERR_SOLVER;
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "bs_orth kernels");
    // H_b -> M_i H_b M_j^T, blocks in chunks (T holds M_i H_b)
    for (int q0 = 0; q0 < nb; q0 += chunk) {
        const int m = nb - q0 < chunk ? nb - q0 : chunk;
        double **hp = h_ptr + (size_t)6 * q0;     // 6 pointers per block, own region per chunk
        for (int q = 0; q < m; q++) {
            const int i = bi[q0 + q], j = bj[q0 + q];
            double *H = hcc + ((size_t)i * (i + 1) / 2 + j) * nn;
            hp[q] = M + nn * i;                 // GEMM 1: T = M_i H
            hp[m + q] = H;
            hp[2 * m + q] = T + nn * q;
            hp[3 * m + q] = T + nn * q;         // GEMM 2: H = T M_j^T
            hp[4 * m + q] = M + nn * j;
            hp[5 * m + q] = H;
        }
        if ((e = cudaMemcpyAsync(d_ptr, hp, sizeof(double *) * 6 * m, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_fail(e, "bs_orth pointer upload");
        cublasStatus_t b1 = cublasDgemmBatched(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, ns, ns, ns, &one,
                                               (const double *const *)d_ptr, ns, (const double *const *)(d_ptr + m),
                                               ns, &zero, d_ptr + 2 * m, ns, m);
        cublasStatus_t b2 = cublasDgemmBatched(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, ns, ns, ns, &one,
                                               (const double *const *)(d_ptr + 3 * m), ns,
                                               (const double *const *)(d_ptr + 4 * m), ns, &zero, d_ptr + 5 * m, ns, m);
        if (b1 != CUBLAS_STATUS_SUCCESS || b2 != CUBLAS_STATUS_SUCCESS) {
            set_error("bsrg_bs_orth: block GEMM failed (%d, %d)", (int)b1, (int)b2);
            return BSRG_ERR_SOLVER;
        }
        // the next chunk's pointer upload is stream-ordered after these GEMMs
    }
    cudaEventRecord(c->ev_stage, s);
    return BSRG_OK;
}

extern "C" int bsrg_diag_hd_ipsol(bsrg_ctx *c, int nch, int *ipsol)
{
    using namespace bsrg;
    if (!c || !ipsol || nch < 1) {
        set_error("bsrg_diag_hd_ipsol: bad arguments");
        return BSRG_ERR_ARG;
    }
    if ((int)c->last_ipsol->size() != nch + 1) {
        set_error("bsrg_diag_hd_ipsol: no bsrg_diag_hd of %d channels on this context", nch);
        return BSRG_ERR_ARG;
    }
    std::memcpy(ipsol, c->last_ipsol->data(), sizeof(int) * (nch + 1));
    return BSRG_OK;
}

extern "C" int bsrg_rsol_out(bsrg_ctx *c, int ns, int nch, const int *ipsol, const double *bb, int khm, const double *a,
                             double *v, double *wmat)
{
    using namespace bsrg;
    if (!c || !ipsol || !bb || !a || !wmat || ns < 1 || nch < 1 || khm < 1 || ipsol[0] != 0 || ipsol[nch] != khm) {
        set_error("bsrg_rsol_out: bad arguments");
        return BSRG_ERR_ARG;
    }
    for (int i = 0; i < nch; i++)
        if (ipsol[i + 1] < ipsol[i] || ipsol[i + 1] - ipsol[i] > ns) {
            set_error("bsrg_rsol_out: channel %d has %d solutions (ns %d)", i + 1, ipsol[i + 1] - ipsol[i], ns);
            return BSRG_ERR_ARG;
        }
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    cudaError_t e;
    const double one = 1.0, zero = 0.0;
    if (v) {
        const int nhm = nch * ns;
        for (int i = 0; i < nch; i++) {
            const int m = ipsol[i + 1] - ipsol[i];
            cublasStatus_t bs;
            if (m == 0) {
                if ((e = cudaMemset2DAsync(v + (size_t)i * ns, sizeof(double) * nhm, 0, sizeof(double) * ns, khm, s)) !=
                    cudaSuccess)
                    return cuda_fail(e, "rsol_out");
                continue;
            }
            bs = cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, ns, khm, m, &one, bb + (size_t)i * ns * ns, ns,
                             a + ipsol[i], khm, &zero, v + (size_t)i * ns, nhm);
            if (bs != CUBLAS_STATUS_SUCCESS) {
                set_error("bsrg_rsol_out: GEMM failed (%d)", (int)bs);
                return BSRG_ERR_SOLVER;
            }
        }
        const size_t nw = (size_t)nch * khm;
        last_rows_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(ns, nch, khm, v, wmat);
    } else {
        int rc = ctx_reserve(c, sizeof(int) * (nch + 1) + 256);
        if (rc != BSRG_OK) return rc;
        if ((rc = ctx_reserve_pinned(c, sizeof(int) * (nch + 1))) != BSRG_OK) return rc;
        if ((e = cudaEventSynchronize(c->ev_stage)) != cudaSuccess) return cuda_fail(e, "rsol_out staging");
        std::memcpy(c->pinned, ipsol, sizeof(int) * (nch + 1));
        int *d_ip = (int *)c->ws;
        if ((e = cudaMemcpyAsync(d_ip, c->pinned, sizeof(int) * (nch + 1), cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_fail(e, "rsol_out upload");
        cudaEventRecord(c->ev_stage, s);
        surface_amplitude_kernel<<<khm, 256, 0, s>>>(ns, nch, d_ip, bb, khm, a, wmat);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "rsol_out");
    return BSRG_OK;
}
