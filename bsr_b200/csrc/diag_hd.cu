// bsr_hd's diagonalisation of one partial wave on the GPU.
//
// Reference: src/bsr/BSR_HD3/diag_hd.f90 for the case the assembly produces,
// an overlap S = blockdiag(sb) (diag_ovl /= 0, "reduced to a STANDARD
// eigenvalue problem", :68-71):
//   1. per channel, drop the first l+1 splines (l capped at ks-2, :83) and the
//      last one if itype = -1, DSYGV('V','U') of (H_ii, S_ii) (:82-111);
//      keep eigenpairs with w <= Edmax (if Edmax /= 0) and |w| >= Egap;
//   2. A = diag(bval) + bb_i^T H_ij bb_j for every stored off-diagonal block
//      (:188-219);
//   3. DSYEV('V','L') of A (:312, LAPACK_calls.f90:54).
// Step 1 runs the library's batched channel solves (chan_eig.cu; cuSOLVER's
// batched path as the fallback), the filter and compaction run on
// the device (one small host read of the per-channel counts fixes khm), step 2
// is two batched FP64 tensor-core GEMMs over all blocks (dgemm.cu), step 3 is
// cuSOLVER's syevd, followed by the FP64 Rayleigh-quotient refinement of every
// eigenpair (refine.cu) when eigenvectors are computed.
#include <algorithm>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "dgemm.h"

namespace bsrg {

// AA[ich](r,c) = H_ii(s0+r, s0+c), CC[ich](r,c) = sb(s0+r, s0+c), leading dimension ns
__global__ void extract_channel_kernel(int ns, int ks, const int *__restrict__ s0v, const int *__restrict__ nsolv,
                                       const double *__restrict__ hcc, const double *__restrict__ sb,
                                       double *AA, double *CC)
{
    int ich = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ns) return;
    int r = tid % ns, c = tid / ns;
    int s0 = s0v[ich], n = nsolv[ich];
    size_t o = (size_t)ich * ns * ns + tid;
    if (r >= n || c >= n) { AA[o] = 0.0; CC[o] = 0.0; return; }
    int i = s0 + r, j = s0 + c;
    const double *H = hcc + ((size_t)(ich + 1) * (ich + 2) / 2 - 1) * ns * ns;
    AA[o] = H[i + (size_t)ns * j];
    int hi = i > j ? i : j, lo = i > j ? j : i;
    double sv = 0.0;
    if (hi - lo < ks) sv = sb[hi + (size_t)ns * (lo - hi + ks - 1)];
    CC[o] = sv;
}

// Padded copies for the batched channel solves (all channels in one batch of
// uniform size n_pad, leading dimension ns):
//   AG[ich] = diag(H_ii restricted to rows/cols s0.., 0)
//   LG[q]   = diag(S restricted likewise, I) for each distinct restriction q
// After the reduction to standard form C = L^-1 H L^-T, pad_shift_kernel puts
// mu = 2 ||C||_F + 1 on the padded diagonal: above every eigenvalue of the
// channel block (|lambda| <= ||C||_2 <= ||C||_F), so the padding's eigenpairs
// sort last, the physical eigenvectors have exactly zero padded components, and
// the padded matrix keeps the channel's own scale (a much larger mu would
// drag the eigensolver's norm-relative tolerances with it).

__global__ void extract_padded_kernel(int ns, int npad, const int *__restrict__ s0v, const int *__restrict__ nsolv,
                                      const double *__restrict__ hcc, double *AG)
{
    int ich = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * npad) return;
    int r = tid % ns, c = tid / ns;
    int n = nsolv[ich], s0 = s0v[ich];
    const double *H = hcc + ((size_t)(ich + 1) * (ich + 2) / 2 - 1) * ns * ns;
    double v = 0.0;
    if (r < n && c < n) v = H[(s0 + r) + (size_t)ns * (s0 + c)];
    AG[(size_t)ich * ns * npad + tid] = v;
}

__global__ void pad_shift_kernel(int ns, int npad, const int *__restrict__ nsolv, double *AG)
{
    int ich = blockIdx.x, n = nsolv[ich];
    double *C = AG + (size_t)ich * ns * npad;
    double ss = 0.0;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        double v = C[(q % n) + (size_t)ns * (q / n)];
        ss += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    __shared__ double part[32];
    __shared__ double mu;
    if (threadIdx.x % 32 == 0) part[threadIdx.x / 32] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) t += part[w];
        mu = 2.0 * sqrt(t) + 1.0;
    }
    __syncthreads();
    for (int r = n + threadIdx.x; r < npad; r += blockDim.x) C[r + (size_t)ns * r] = mu;
}

__global__ void extract_padded_overlap_kernel(int ns, int ks, int npad, const int *__restrict__ gs0,
                                              const int *__restrict__ gn, const double *__restrict__ sb, double *LG)
{
    int q = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * npad) return;
    int r = tid % ns, c = tid / ns;
    int n = gn[q], s0 = gs0[q];
    double v = 0.0;
    if (r < n && c < n) {
        int i = s0 + r, j = s0 + c, hi = i > j ? i : j, lo = i > j ? j : i;
        if (hi - lo < ks) v = sb[hi + (size_t)ns * (lo - hi + ks - 1)];
    } else if (r == c && r < npad) v = 1.0;
    LG[(size_t)q * ns * npad + tid] = v;
}

// channel solutions back to the per-channel slots read by keep_count/compact
__global__ void scatter_back_kernel(int ns, int npad, const int *__restrict__ nsolv, const double *__restrict__ AG,
                                    const double *__restrict__ WG, double *AA, double *Wv)
{
    int ich = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int n = nsolv[ich];
    if (tid >= ns * n) return;
    AA[(size_t)ich * ns * ns + tid] = AG[(size_t)ich * ns * npad + tid];
    if (tid < n) Wv[(size_t)ich * ns + tid] = WG[(size_t)ich * npad + tid];
}

__global__ void keep_count_kernel(int ns, int nch, const int *__restrict__ nsolv, const double *__restrict__ W,
                                  double edmax, double egap, int *counts)
{
    int ich = blockIdx.x;
    if (ich >= nch) return;
    int n = nsolv[ich], cnt = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double w = W[(size_t)ich * ns + i];
        bool keep = !(edmax != 0.0 && w > edmax) && !(egap > 0.0 && fabs(w) < egap);
        cnt += keep;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    __shared__ int part[32];
    if (threadIdx.x % 32 == 0) part[threadIdx.x / 32] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int q = 0; q < (int)(blockDim.x + 31) / 32; q++) s += part[q];
        counts[ich] = s;
    }
}

// bval[ipsol[ich]+q] and BB[ich](:, q) for the q-th kept solution (ascending order kept)
__global__ void compact_kernel(int ns, const int *__restrict__ s0v, const int *__restrict__ nsolv,
                               const int *__restrict__ ipsol, const double *__restrict__ W,
                               const double *__restrict__ AA, double edmax, double egap, double *bval, double *BB)
{
    int ich = blockIdx.x;
    __shared__ int rank[1024];
    int n = nsolv[ich], s0 = s0v[ich];
    if (threadIdx.x == 0) {
        int q = 0;
        for (int i = 0; i < n; i++) {
            double w = W[(size_t)ich * ns + i];
            bool keep = !(edmax != 0.0 && w > edmax) && !(egap > 0.0 && fabs(w) < egap);
            rank[i] = keep ? q++ : -1;
        }
    }
    __syncthreads();
    double *B = BB + (size_t)ich * ns * ns;
    // zero the whole padded block first
    for (int q = threadIdx.x; q < ns * ns; q += blockDim.x) B[q] = 0.0;
    __syncthreads();
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        int r = q % n, i = q / n;
        int dst = rank[i];
        if (dst < 0) continue;
        B[(s0 + r) + (size_t)ns * dst] = AA[(size_t)ich * ns * ns + r + (size_t)ns * i];
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (rank[i] >= 0) bval[ipsol[ich] + rank[i]] = W[(size_t)ich * ns + i];
}

struct BlockMap { int ic, jc; };   // 0-based channels, ic > jc

__global__ void scatter_blocks_kernel(int ns, long lda, const BlockMap *__restrict__ bm, const int *__restrict__ ipsol,
                                      const double *__restrict__ T, double *A)
{
    int b = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ns) return;
    int r = tid % ns, c = tid / ns;
    BlockMap m = bm[b];
    int nr = ipsol[m.ic + 1] - ipsol[m.ic], nc = ipsol[m.jc + 1] - ipsol[m.jc];
    if (r >= nr || c >= nc) return;
    A[(size_t)(ipsol[m.ic] + r) + (size_t)lda * (ipsol[m.jc] + c)] = T[(size_t)b * ns * ns + tid];
}

__global__ void fill_diag_kernel(long n, double v, double *A)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) A[i + n * i] = v;
}

__global__ void set_diag_kernel(long n, const double *__restrict__ bval, double *A)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) A[i + n * i] = bval[i];
}

struct ChannelGroups {
    std::vector<int> gs0, gn;                 // first row and size of each group
    std::vector<std::vector<int>> members;    // channels of each group
};

static ChannelGroups group_channels(const std::vector<int> &s0v, const std::vector<int> &nsolv)
{
    ChannelGroups G;
    for (size_t ich = 0; ich < s0v.size(); ich++) {
        int q = -1;
        for (size_t k = 0; k < G.gs0.size(); k++)
            if (G.gs0[k] == s0v[ich] && G.gn[k] == nsolv[ich]) { q = (int)k; break; }
        if (q < 0) {
            q = (int)G.gs0.size();
            G.gs0.push_back(s0v[ich]);
            G.gn.push_back(nsolv[ich]);
            G.members.emplace_back();
        }
        G.members[q].push_back((int)ich);
    }
    return G;
}

// device bytes the batched channel solves take from the arena (0 if unavailable)
static size_t chan_batched_bytes(bsrg_ctx *c, cusolverDnParams_t params, int ns, const std::vector<int> &s0v,
                                 const std::vector<int> &nsolv)
{
    ChannelGroups G = group_channels(s0v, nsolv);
    int nch = (int)s0v.size(), ng = (int)G.gs0.size();
    int npad = *std::max_element(nsolv.begin(), nsolv.end());
    size_t d1 = 0, h1 = 0;
    if (cusolverDnXsyevBatched_bufferSize(c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, npad,
                                          CUDA_R_64F, nullptr, ns, CUDA_R_64F, nullptr, CUDA_R_64F, &d1, &h1,
                                          (int64_t)nch) != CUSOLVER_STATUS_SUCCESS)
        return 0;
    size_t bytes = 0;
    auto add = [&](size_t b) { bytes += ((b + 255) & ~(size_t)255) + 256; };
    add(sizeof(double) * (size_t)ns * npad * nch);   // AG
    add(sizeof(double) * (size_t)npad * nch);        // WG
    add(sizeof(double) * (size_t)ns * npad * ng);    // LG
    add(d1 + 16);
    add(sizeof(int) * ng * 2);
    add(sizeof(double *) * (2 * (size_t)nch + ng));
    add(sizeof(int) * (nch + ng));
    return bytes;
}

// Is cuSOLVER's batched symmetric eigensolver usable for these channel sizes?
static bool chan_batched_ok(bsrg_ctx *c, cusolverDnParams_t params, int ns, const std::vector<int> &nsolv)
{
    if (getenv("BSRG_CHANNEL_SYGVD")) return false;
    size_t dws = 0, hws = 0;
    int n = *std::max_element(nsolv.begin(), nsolv.end());
    cusolverStatus_t st = cusolverDnXsyevBatched_bufferSize(c->solver, params, CUSOLVER_EIG_MODE_VECTOR,
                                                            CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, nullptr, ns,
                                                            CUDA_R_64F, nullptr, CUDA_R_64F, &dws, &hws, 1);
    return st == CUSOLVER_STATUS_SUCCESS;
}

// The batched channel solves.  Writes eigenvectors (normalised to x^T S x = 1)
// into AA[ich] (ld ns) and eigenvalues into Wv[ich*ns], like sygvd would: one
// batched Cholesky of the distinct restricted overlaps (DPOTRF), two batched
// triangular solves (DSYGST), one batched symmetric eigensolve of all channels
// (DSYEV) and the batched back-transform x = L^-T y.
static int solve_channels_batched(bsrg_ctx *c, cusolverDnParams_t params, const bsrg_basis *b, const double *hcc,
                                  int nch, const std::vector<int> &s0v, const std::vector<int> &nsolv,
                                  const int *d_s0, const int *d_nsol, double *AA, double *Wv, int *d_info,
                                  Arena &ar)
{
    const int ns = b->ns, ks = b->ks;
    cudaStream_t s = c->stream;
    cudaError_t e;
    ChannelGroups G = group_channels(s0v, nsolv);
    const int ng = (int)G.gs0.size();
    const int npad = *std::max_element(nsolv.begin(), nsolv.end());
    size_t dws = 0, hws = 0;
    if (cusolverDnXsyevBatched_bufferSize(c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, npad,
                                          CUDA_R_64F, nullptr, ns, CUDA_R_64F, nullptr, CUDA_R_64F, &dws, &hws,
                                          (int64_t)nch) != CUSOLVER_STATUS_SUCCESS) {
        set_error("diag_hd: syevBatched_bufferSize failed");
        return BSRG_ERR_SOLVER;
    }
    double *AG = ar.take<double>((size_t)ns * npad * nch), *WG = ar.take<double>((size_t)npad * nch);
    double *LG = ar.take<double>((size_t)ns * npad * ng);
    void *swork = ar.take<char>(dws + 16);
    int *d_gs0 = ar.take<int>(ng), *d_gn = ar.take<int>(ng);
    double **d_ptr = ar.take<double *>(2 * (size_t)nch + ng);    // L per channel | A per channel | L per group
    int *d_binfo = ar.take<int>((size_t)nch + ng);               // syev info, then potrf info
    if (ar.off > ar.cap) { set_error("diag_hd: workspace too small for the batched channel solves"); return BSRG_ERR_NOMEM; }
    std::vector<char> hwork(hws + 16);
    std::vector<double *> hptr(2 * (size_t)nch + ng);
    std::vector<int> grp(nch);
    for (int q = 0; q < ng; q++)
        for (int ich : G.members[q]) grp[ich] = q;
    for (int ich = 0; ich < nch; ich++) {
        hptr[ich] = LG + (size_t)grp[ich] * ns * npad;
        hptr[nch + ich] = AG + (size_t)ich * ns * npad;
    }
    for (int q = 0; q < ng; q++) hptr[2 * (size_t)nch + q] = LG + (size_t)q * ns * npad;
    if ((e = cudaMemcpyAsync(d_gs0, G.gs0.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_gn, G.gn.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_ptr, hptr.data(), sizeof(double *) * hptr.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(e, "diag_hd batched upload");
    {
        dim3 g((unsigned)((ns * npad + 127) / 128), nch);
        extract_padded_kernel<<<g, 128, 0, s>>>(ns, npad, d_s0, d_nsol, hcc, AG);
        dim3 g2((unsigned)((ns * npad + 127) / 128), ng);
        extract_padded_overlap_kernel<<<g2, 128, 0, s>>>(ns, ks, npad, d_gs0, d_gn, b->sb, LG);
    }
    double **Lp = d_ptr, **Ap = d_ptr + nch, **Lg = d_ptr + 2 * nch;
    if (cusolverDnDpotrfBatched(c->solver, CUBLAS_FILL_MODE_LOWER, npad, Lg, ns, d_binfo + nch, ng) !=
        CUSOLVER_STATUS_SUCCESS) {
        set_error("diag_hd: potrfBatched failed to launch");
        return BSRG_ERR_SOLVER;
    }
    const double one = 1.0;
    cublasStatus_t b1 = cublasDtrsmBatched(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                                           CUBLAS_DIAG_NON_UNIT, npad, npad, &one, (const double *const *)Lp, ns, Ap,
                                           ns, nch);
    cublasStatus_t b2 = cublasDtrsmBatched(c->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                                           CUBLAS_DIAG_NON_UNIT, npad, npad, &one, (const double *const *)Lp, ns, Ap,
                                           ns, nch);
    if (b1 != CUBLAS_STATUS_SUCCESS || b2 != CUBLAS_STATUS_SUCCESS) {
        set_error("diag_hd: trsmBatched failed (%d, %d)", (int)b1, (int)b2);
        return BSRG_ERR_SOLVER;
    }
    pad_shift_kernel<<<nch, 256, 0, s>>>(ns, npad, d_nsol, AG);
    if (cusolverDnXsyevBatched(c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, npad, CUDA_R_64F,
                               AG, ns, CUDA_R_64F, WG, CUDA_R_64F, swork, dws, hwork.data(), hws, d_binfo,
                               nch) != CUSOLVER_STATUS_SUCCESS) {
        set_error("diag_hd: syevBatched failed to launch");
        return BSRG_ERR_SOLVER;
    }
    cublasStatus_t b3 = cublasDtrsmBatched(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                                           CUBLAS_DIAG_NON_UNIT, npad, npad, &one, (const double *const *)Lp, ns, Ap,
                                           ns, nch);
    if (b3 != CUBLAS_STATUS_SUCCESS) {
        set_error("diag_hd: trsmBatched (back-transform) failed (%d)", (int)b3);
        return BSRG_ERR_SOLVER;
    }
    dim3 g((unsigned)((ns * npad + 127) / 128), nch);
    scatter_back_kernel<<<g, 128, 0, s>>>(ns, npad, d_nsol, AG, WG, AA, Wv);
    // cuSOLVER needs the host workspace alive until the work is done; check the infos here
    std::vector<int> hinfo((size_t)nch + ng);
    if ((e = cudaMemcpyAsync(hinfo.data(), d_binfo, sizeof(int) * (nch + ng), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "diag_hd batched info");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "diag_hd batched channel solves");
    for (int q = 0; q < ng; q++)
        if (hinfo[nch + q] != 0) {
            set_error("BSR_HD: channel diagonalization failed, overlap of channel = %d not positive definite (info %d)",
                      G.members[q][0] + 1, hinfo[nch + q]);
            return BSRG_ERR_INFO;
        }
    for (int ich = 0; ich < nch; ich++)
        if (hinfo[ich] != 0) {
            set_error("BSR_HD: channel diagonalization failed, channel = %d (info %d)", ich + 1, hinfo[ich]);
            return BSRG_ERR_INFO;
        }
    if ((e = cudaMemsetAsync(d_info, 0, sizeof(int) * nch, s)) != cudaSuccess) return cuda_fail(e, "diag_hd info");
    return cuda_fail(cudaGetLastError(), "diag_hd batched channel solves");
}

}  // namespace bsrg

using namespace bsrg;

// smallest dense problem (by its row bound) for which diag_hd uses the library's eigensolver by
// default: measured against cuSOLVER's syevd on a B200, 399 vs 421 ms at 7810 rows, 258 vs 228 ms
// at 6000 and 154 vs 114 ms at 4500
constexpr int kOwnEigMin = 7000;

// scc == NULL: the block-diagonal overlap (diag_ovl /= 0); otherwise the generalized
// branch with the channel-channel overlap blocks of scc (diag_ovl = 0)
static int diag_hd_impl(bsrg_ctx *c, const bsrg_basis *b, int nch, const int *lch, const double *hcc,
                        const double *scc, int itype, int ilzero, int ibzero, double edmax, double egap,
                        int want_vectors, double *eval, int *khm_out, double *vecs, double *bbout)
{
    if (!c || !b || !lch || !hcc || !eval || !khm_out) {
        set_error("diag_hd: null argument");
        return BSRG_ERR_ARG;
    }
    if (nch < 1) { set_error("diag_hd: nch=%d", nch); return BSRG_ERR_ARG; }
    const int ns = b->ns, ks = b->ks;
    if (ns > 1024) { set_error("diag_hd: ns=%d above 1024", ns); return BSRG_ERR_ARG; }
    cudaStream_t s = c->stream;
    cudaError_t e;
    // ---- per-channel geometry (diag_hd.f90:83-86) ----
    std::vector<int> s0v(nch), nsolv(nch);
    for (int ich = 0; ich < nch; ich++) {
        int l = lch[ich];
        if (l > ks - 2) l = ks - 2;
        if (ilzero == 0) l = 0;
        int i1 = l + 2, i2 = ns;
        if (itype == -1) i2 = ns - ibzero;
        s0v[ich] = i1 - 1;
        nsolv[ich] = i2 - i1 + 1;
        if (nsolv[ich] < 1) { set_error("diag_hd: channel %d has no solutions", ich + 1); return BSRG_ERR_ARG; }
    }
    // The refined form (default with eigenvectors) also transforms the diagonal
    // blocks, bb_i^T H_ii bb_i, instead of taking diag(bval): the two are equal in
    // exact arithmetic (diag_hd.f90:188-219 stores diag(bval)), but explicitly
    // formed blocks keep the channel solver's rounding (~eps ||H_ii||) out of
    // the eigenvalues, which the Rayleigh quotients below then resolve.
    const bool refine = want_vectors && c->refine;
    const char *eig_env = getenv("BSRG_EIG");
    // the library's two-stage eigensolver (syevd2.cu) or cuSOLVER's syevd: BSRG_EIG=own or =lib
    // chooses, else the context's setting; by default the library's from kOwnEigMin rows up (where
    // it was measured faster)
    int khm_bound = 0;
    for (int ich = 0; ich < nch; ich++) khm_bound += nsolv[ich];
    const bool own_eig = want_vectors && khm_bound <= 10240 &&
                         (eig_env ? strcmp(eig_env, "own") == 0
                                  : (c->eig_mode == 1 || (c->eig_mode == 0 && khm_bound >= kOwnEigMin)));
    std::vector<BlockMap> bmap;
    for (int ic = 1; ic < nch; ic++)
        for (int jc = 0; jc < ic; jc++) bmap.push_back({ic, jc});
    if (refine)
        for (int ic = 0; ic < nch; ic++) bmap.push_back({ic, ic});
    const int nb = (int)bmap.size();
    // ---- workspace: phase 1 ----
    size_t nn = (size_t)ns * ns;
    int lwork1 = 0;
    if (cusolverDnDsygvd_bufferSize(c->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER,
                                    ns, nullptr, ns, nullptr, ns, nullptr, &lwork1) != CUSOLVER_STATUS_SUCCESS) {
        set_error("diag_hd: sygvd_bufferSize failed");
        return BSRG_ERR_SOLVER;
    }
    // worst case khm for sizing the dense phase up front
    int khm_max = 0;
    for (int ich = 0; ich < nch; ich++) khm_max += nsolv[ich];
    cusolverDnParams_t params;
    if (cusolverDnCreateParams(&params) != CUSOLVER_STATUS_SUCCESS) {
        set_error("diag_hd: cusolverDnCreateParams failed");
        return BSRG_ERR_SOLVER;
    }
    cusolverEigMode_t jobz = want_vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
    size_t dws = 0, hws = 0;
    if (cusolverDnXsyevd_bufferSize(c->solver, params, jobz, CUBLAS_FILL_MODE_LOWER, khm_max, CUDA_R_64F, nullptr,
                                    khm_max, CUDA_R_64F, nullptr, CUDA_R_64F, &dws, &hws) != CUSOLVER_STATUS_SUCCESS) {
        cusolverDnDestroyParams(params);
        set_error("diag_hd: syevd_bufferSize failed");
        return BSRG_ERR_SOLVER;
    }
    size_t need = 0;
    auto add = [&](size_t bytes) { need += ((bytes + 255) & ~(size_t)255) + 256; };
    add(sizeof(int) * nch * 3 + 64);      // s0, nsol, counts
    add(sizeof(int) * (nch + 1));         // ipsol
    add(sizeof(int) * (nch + 1));         // infos
    add(sizeof(double) * nn * nch * 3);   // AA, CC, BB
    add(sizeof(double) * (size_t)ns * nch * 2);  // W, bval
    add(sizeof(double) * (size_t)lwork1);
    add(sizeof(BlockMap) * std::max(nb, 1));
    add(sizeof(double *) * std::max(nb, 1) * 6);
    add(sizeof(double) * nn * std::max(nb, 1) * 2);   // Wt, T
    if (!vecs) add(sizeof(double) * (size_t)khm_max * khm_max);
    add(dws + 16);
    // the mixed-precision form's A V from 8-bit digits (its K limit: the FP64 GEMM beyond)
    const bool oz_refine = refine && c->precision == 1 && khm_max <= BSRG_OZAKI_KMAX;
    const size_t oz_bytes = oz_refine ? ozaki_ws_bytes(khm_max, khm_max, khm_max, 8) : 0;
    if (refine) {
        add(sizeof(double) * refine_workspace_doubles(khm_max));   // mirrored A, then the tile partial sums
        add(sizeof(int) * 4);
        if (oz_refine) add(oz_bytes);
    }
    if (own_eig) add(sizeof(double) * syevd2_workspace_doubles(khm_max));
    const bool gen = scc != nullptr;
    int nbo = 0;                          // off-diagonal overlap blocks to transform
    if (gen) {
        nbo = nch * (nch - 1) / 2;
        add(sizeof(double) * (size_t)khm_max * khm_max * 2);       // C (overlap), then the DSYGST transpose
        add(sizeof(double) * chol_workspace_doubles(khm_max));
        add(sizeof(int) * 4);
    }
    size_t batched_bytes = chan_batched_bytes(c, params, ns, s0v, nsolv);
    add(batched_bytes);
    // the library's own channel solves (chan_eig.cu); BSRG_CHANNEL_LIB selects cuSOLVER's batched path
    const int npad = *std::max_element(nsolv.begin(), nsolv.end());
    const bool own_chan = !getenv("BSRG_CHANNEL_LIB") && !getenv("BSRG_CHANNEL_SYGVD") &&
                          chan_own_ok(ns, ks, npad, c->device);
    if (own_chan) {
        add(sizeof(double) * chan_own_workspace_doubles(nch, npad, ks));
        add(sizeof(int) * 4);
    }
    int rc = ctx_reserve(c, need);
    if (rc != BSRG_OK) { cusolverDnDestroyParams(params); return rc; }
    // pinned staging layout (ints): s0 | nsol | info | cnt | ipsol | final info, then block maps and pointers
    const size_t o_s0 = 0, o_nsol = nch, o_info = 2 * (size_t)nch, o_cnt = 3 * (size_t)nch, o_ip = 4 * (size_t)nch,
                 o_fin = 5 * (size_t)nch + 1;
    size_t o_bm_bytes = ((o_fin + 2) * sizeof(int) + 15) & ~(size_t)15;
    size_t o_ptr_bytes = (o_bm_bytes + sizeof(BlockMap) * nb + 15) & ~(size_t)15;
    const size_t o_dc_bytes = (o_ptr_bytes + sizeof(double *) * nb * 6 + 64 + 255) & ~(size_t)255;
    rc = ctx_reserve_pinned(c, o_dc_bytes + (own_eig ? dc_pinned_bytes(khm_max) : 0) + 64);
    if (rc != BSRG_OK) { cusolverDnDestroyParams(params); return rc; }
    Arena ar{(char *)c->ws, 0, c->ws_bytes};
    int *d_s0 = ar.take<int>(nch), *d_nsol = ar.take<int>(nch), *d_cnt = ar.take<int>(nch);
    int *d_ipsol = ar.take<int>(nch + 1), *d_info = ar.take<int>(nch + 1);
    double *AA = ar.take<double>(nn * nch), *CC = ar.take<double>(nn * nch), *BB = ar.take<double>(nn * nch);
    double *Wv = ar.take<double>((size_t)ns * nch), *bval = ar.take<double>((size_t)ns * nch);
    double *work1 = ar.take<double>(std::max(lwork1, 1));
    BlockMap *d_bm = ar.take<BlockMap>(std::max(nb, 1));
    double **d_ptrs = ar.take<double *>((size_t)std::max(nb, 1) * 6);
    double *Wt = ar.take<double>(nn * std::max(nb, 1)), *T = ar.take<double>(nn * std::max(nb, 1));
    double *Abuf = vecs ? nullptr : ar.take<double>((size_t)khm_max * khm_max);
    void *dwork = ar.take<char>(dws + 16);
    double *Fsym = refine ? ar.take<double>(refine_workspace_doubles(khm_max)) : nullptr;
    int *d_rflag = refine ? ar.take<int>(4) : nullptr;
    char *oz_ws = oz_refine ? ar.take<char>(oz_bytes) : nullptr;
    double *eig_ws = own_eig ? ar.take<double>(syevd2_workspace_doubles(khm_max)) : nullptr;
    double *chan_ws = own_chan ? ar.take<double>(chan_own_workspace_doubles(nch, npad, ks)) : nullptr;
    double *Cov = gen ? ar.take<double>((size_t)khm_max * khm_max) : nullptr;
    double *Tgst = gen ? ar.take<double>((size_t)khm_max * khm_max) : nullptr;
    double *chol_ws = gen ? ar.take<double>(chol_workspace_doubles(khm_max)) : nullptr;
    int *d_cinfo = gen ? ar.take<int>(4) : nullptr;
    int *d_cflag = own_chan ? ar.take<int>(4) : nullptr;
    int *hi = (int *)c->pinned;
    std::memcpy(hi + o_s0, s0v.data(), sizeof(int) * nch);
    std::memcpy(hi + o_nsol, nsolv.data(), sizeof(int) * nch);
    if ((e = cudaMemcpyAsync(d_s0, hi + o_s0, sizeof(int) * nch, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_nsol, hi + o_nsol, sizeof(int) * nch, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
        cusolverDnDestroyParams(params);
        return cuda_fail(e, "diag_hd upload");
    }
    // ---- 1. channel problems ----
    // Channels with the same l share the restricted overlap S_l.  Per group:
    // DPOTRF(S_l) once, then for all its channels at once DSYGST as two
    // batched triangular solves, a batched DSYEV and the back-transform
    // x = L^-T y (the steps of LAPACK's DSYGV).  If the batched eigensolver is
    // not available in the loaded cuSOLVER, each channel goes through sygvd.
    stage_begin(c, 4);
    bool batched = batched_bytes > 0 && chan_batched_ok(c, params, ns, nsolv);
    int chan_launches = batched ? 5 : 2;
    bool own_done = false;
    if (own_chan) {
        // the own kernels; if the eigenvectors of a channel come out far from orthonormal
        // (eigenvalues equal to working precision), the library path below redoes all channels
        int rco = chan_own_solve(c, b, hcc, nch, npad, d_s0, d_nsol, AA, Wv, d_info, chan_ws, d_cflag);
        if (rco != BSRG_OK) { cusolverDnDestroyParams(params); return rco; }
        int hf[2] = {0, 0};
        if ((e = cudaMemcpyAsync(hf, d_cflag, sizeof(hf), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            cusolverDnDestroyParams(params);
            return cuda_fail(e, "diag_hd channel solves");
        }
        own_done = hf[0] == 0 && hf[1] == 0;
        chan_launches = 8;
        if (!own_done) c->chan_fallbacks++;
    }
    if (own_done) {
    } else if (batched) {
        int rcb = solve_channels_batched(c, params, b, hcc, nch, s0v, nsolv, d_s0, d_nsol, AA, Wv, d_info, ar);
        if (rcb != BSRG_OK) { cusolverDnDestroyParams(params); return rcb; }
    } else {
        {
            dim3 g((unsigned)((nn + 127) / 128), nch);
            extract_channel_kernel<<<g, 128, 0, s>>>(ns, ks, d_s0, d_nsol, hcc, b->sb, AA, CC);
        }
        for (int ich = 0; ich < nch; ich++) {
            cusolverStatus_t st = cusolverDnDsygvd(c->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                   CUBLAS_FILL_MODE_UPPER, nsolv[ich], AA + nn * ich, ns, CC + nn * ich,
                                                   ns, Wv + (size_t)ns * ich, work1, lwork1, d_info + ich);
            if (st != CUSOLVER_STATUS_SUCCESS) {
                cusolverDnDestroyParams(params);
                set_error("diag_hd: sygvd failed to launch for channel %d (status %d)", ich + 1, (int)st);
                return BSRG_ERR_SOLVER;
            }
        }
    }
    keep_count_kernel<<<nch, 256, 0, s>>>(ns, nch, d_nsol, Wv, edmax, egap, d_cnt);
    stage_end(c, 4, chan_launches);     // own kernels (the library path: extracts, pad shift, scatter-back)
    if ((e = cudaMemcpyAsync(hi + o_info, d_info, sizeof(int) * nch, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hi + o_cnt, d_cnt, sizeof(int) * nch, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
        cusolverDnDestroyParams(params);
        return cuda_fail(e, "diag_hd readback");
    }
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
        cusolverDnDestroyParams(params);
        return cuda_fail(e, "diag_hd channel solves");
    }
    for (int ich = 0; ich < nch; ich++)
        if (hi[o_info + ich] != 0) {
            cusolverDnDestroyParams(params);
            set_error("BSR_HD: channel diagonalization failed, channel = %d (info %d)", ich + 1, hi[o_info + ich]);
            return BSRG_ERR_INFO;
        }
    std::vector<int> ipsol(nch + 1, 0);
    for (int ich = 0; ich < nch; ich++) ipsol[ich + 1] = ipsol[ich] + hi[o_cnt + ich];
    const int khm = ipsol[nch];
    *khm_out = khm;
    *c->last_ipsol = ipsol;
    if (khm == 0) {
        cusolverDnDestroyParams(params);
        set_error("diag_hd: no channel solutions survive the filter");
        return BSRG_ERR_INFO;
    }
    const size_t dws_cap = dws;
    if (cusolverDnXsyevd_bufferSize(c->solver, params, jobz, CUBLAS_FILL_MODE_LOWER, khm, CUDA_R_64F, nullptr, khm,
                                    CUDA_R_64F, nullptr, CUDA_R_64F, &dws, &hws) != CUSOLVER_STATUS_SUCCESS ||
        dws > dws_cap) {
        cusolverDnDestroyParams(params);
        set_error("diag_hd: syevd_bufferSize failed");
        return BSRG_ERR_SOLVER;
    }
    size_t asz = (size_t)khm * khm;
    double *A = vecs ? vecs : Abuf;
    std::vector<char> hwork(hws + 16);
    // ---- compaction ----
    int *h_ip = hi + o_ip;
    std::memcpy(h_ip, ipsol.data(), sizeof(int) * (nch + 1));
    BlockMap *h_bm = (BlockMap *)((char *)c->pinned + o_bm_bytes);
    if (nb > 0) std::memcpy(h_bm, bmap.data(), sizeof(BlockMap) * nb);
    double **h_ptrs = (double **)((char *)c->pinned + o_ptr_bytes);
    for (int q = 0; q < nb; q++) {
        const BlockMap &m = bmap[q];
        h_ptrs[q] = (double *)(hcc + ((size_t)(m.ic + 1) * m.ic / 2 + m.jc) * nn);   // H_ij, i = ic+1 (1-based), j <= i
        h_ptrs[nb + q] = BB + nn * m.jc;
        h_ptrs[2 * nb + q] = Wt + nn * q;
        h_ptrs[3 * nb + q] = BB + nn * m.ic;
        h_ptrs[4 * nb + q] = T + nn * q;
        // overlap block S_ij of the generalized branch (the first nbo entries: the off-diagonal pairs)
        h_ptrs[5 * nb + q] = (gen && q < nbo) ? (double *)(scc + ((size_t)(m.ic + 1) * m.ic / 2 + m.jc) * nn) : nullptr;
    }
    if ((e = cudaMemcpyAsync(d_ipsol, h_ip, sizeof(int) * (nch + 1), cudaMemcpyHostToDevice, s)) != cudaSuccess) {
        cusolverDnDestroyParams(params);
        return cuda_fail(e, "diag_hd ipsol upload");
    }
    if (nb > 0) {
        if ((e = cudaMemcpyAsync(d_bm, h_bm, sizeof(BlockMap) * nb, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_ptrs, h_ptrs, sizeof(double *) * nb * 6, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
            cusolverDnDestroyParams(params);
            return cuda_fail(e, "diag_hd block upload");
        }
    }
    cudaEventRecord(c->ev_stage, s);
    stage_begin(c, 5);
    compact_kernel<<<nch, 256, 0, s>>>(ns, d_s0, d_nsol, d_ipsol, Wv, AA, edmax, egap, bval, BB);
    // ---- 2. A = diag(bval) + bb^T H_ij bb ----
    if ((e = cudaMemsetAsync(A, 0, sizeof(double) * asz, s)) != cudaSuccess) {
        cusolverDnDestroyParams(params);
        return cuda_fail(e, "memset A");
    }
    if (!refine) set_diag_kernel<<<(khm + 255) / 256, 256, 0, s>>>(khm, bval, A);
    if (nb > 0) {
        double **pH = d_ptrs, **pBj = d_ptrs + nb, **pW = d_ptrs + 2 * nb, **pBi = d_ptrs + 3 * nb,
               **pT = d_ptrs + 4 * nb;
        // W = H_ij bb_j, then T = bb_i^T W: two batched FP64 tensor-core GEMMs
        DgemmBatch g1{};
        g1.m = ns; g1.n = ns; g1.k = ns;
        g1.lda = ns; g1.ldb = ns; g1.ldc = ns;
        g1.Ap = (const double *const *)pH; g1.Bp = (const double *const *)pBj; g1.Cp = pW;
        g1.alpha = 1.0; g1.beta = 0.0;
        DgemmBatch g2 = g1;
        g2.Ap = (const double *const *)pBi; g2.Bp = (const double *const *)pW; g2.Cp = pT;
        int rg = dgemm_batched(false, false, g1, nb, s);
        if (rg == BSRG_OK) rg = dgemm_batched(true, false, g2, nb, s);
        if (rg != BSRG_OK) { cusolverDnDestroyParams(params); return rg; }
        dim3 g((unsigned)((nn + 127) / 128), nb);
        scatter_blocks_kernel<<<g, 128, 0, s>>>(ns, khm, d_bm, d_ipsol, T, A);
    }
    int t_launches = (nb > 0 ? 4 : 1) + (refine ? 0 : 1);   // compact, [set_diag], 2 GEMMs, scatter
    c->stage_flops[5] += 4.0 * (double)ns * ns * ns * nb;
    if (gen) {
        // ---- generalized branch: C = I + bb_i^T S_ij bb_j (diag_hd.f90:127-186), DPOTRF(C) and
        //      DSYGST(1,'L') of A (:268-284) ----
        if ((e = cudaMemsetAsync(Cov, 0, sizeof(double) * asz, s)) != cudaSuccess ||
            (e = cudaMemsetAsync(d_cinfo, 0, sizeof(int), s)) != cudaSuccess) {
            cusolverDnDestroyParams(params);
            return cuda_fail(e, "diag_hd overlap");
        }
        fill_diag_kernel<<<(khm + 255) / 256, 256, 0, s>>>(khm, 1.0, Cov);
        t_launches++;
        if (nbo > 0) {
            double **pS = d_ptrs + 5 * nb, **pBj = d_ptrs + nb, **pW = d_ptrs + 2 * nb, **pBi = d_ptrs + 3 * nb,
                   **pT = d_ptrs + 4 * nb;
            DgemmBatch g1{};
            g1.m = ns; g1.n = ns; g1.k = ns;
            g1.lda = ns; g1.ldb = ns; g1.ldc = ns;
            g1.Ap = (const double *const *)pS; g1.Bp = (const double *const *)pBj; g1.Cp = pW;
            g1.alpha = 1.0; g1.beta = 0.0;
            DgemmBatch g2 = g1;
            g2.Ap = (const double *const *)pBi; g2.Bp = (const double *const *)pW; g2.Cp = pT;
            int rg = dgemm_batched(false, false, g1, nbo, s);
            if (rg == BSRG_OK) rg = dgemm_batched(true, false, g2, nbo, s);
            if (rg != BSRG_OK) { cusolverDnDestroyParams(params); return rg; }
            dim3 g((unsigned)((nn + 127) / 128), nbo);
            scatter_blocks_kernel<<<g, 128, 0, s>>>(ns, khm, d_bm, d_ipsol, T, Cov);
            t_launches += 3;
            c->stage_flops[5] += 4.0 * (double)ns * ns * ns * nbo;
        }
        double *Linv = chol_ws, *ctmp = chol_ws + (chol_workspace_doubles(khm_max) - (size_t)khm_max * 128 - 64);
        const size_t ctmp_doubles = (size_t)khm_max * 128 + 64;
        int rg = dpotrf_lower(khm, Cov, khm, Linv, ctmp, d_cinfo, s, &t_launches);
        if (rg == BSRG_OK) rg = mirror_lower(khm, A, khm, s);
        if (rg == BSRG_OK) rg = sygst_lower(khm, A, khm, Cov, khm, Linv, Tgst, ctmp, ctmp_doubles, s, &t_launches);
        if (rg != BSRG_OK) { cusolverDnDestroyParams(params); return rg; }
        t_launches++;
        c->stage_flops[5] += (1.0 / 3.0 + 2.0) * (double)khm * khm * khm;
    }
    stage_end(c, 5, t_launches);
    if (refine) {
        // keep the full symmetric A for the residuals: the eigensolver overwrites A
        stage_begin(c, 8);
        int rr = refine_prepare(khm, A, khm, Fsym, s);
        stage_end(c, 8, 1);
        if (rr != BSRG_OK) { cusolverDnDestroyParams(params); return rr; }
    }
    // ---- 3. eigensolve ----
    stage_begin(c, 6);
    if (own_eig) {
        cusolverDnDestroyParams(params);
        int nlaunch = 0;
        int re = dense_syevd(c, khm, A, khm, eval, A, khm, eig_ws, syevd2_workspace_doubles(khm_max),
                             (char *)c->pinned + o_dc_bytes, c->pinned_bytes - o_dc_bytes, &nlaunch);
        stage_end(c, 6, nlaunch);
        if (re != BSRG_OK) return re;
        if ((e = cudaMemsetAsync(d_info + nch, 0, sizeof(int), s)) != cudaSuccess) return cuda_fail(e, "diag_hd info");
    } else {
        cusolverStatus_t st = cusolverDnXsyevd(c->solver, params, jobz, CUBLAS_FILL_MODE_LOWER, khm, CUDA_R_64F, A,
                                               khm, CUDA_R_64F, eval, CUDA_R_64F, dwork, dws, hwork.data(), hws,
                                               d_info + nch);
        cusolverDnDestroyParams(params);
        stage_end(c, 6, 0);
        if (st != CUSOLVER_STATUS_SUCCESS) {
            set_error("diag_hd: syevd failed to launch (status %d)", (int)st);
            return BSRG_ERR_SOLVER;
        }
    }
    if (refine) {
        // ---- FP64 refinement of the eigenpairs (windowed Rayleigh-Ritz values) ----
        if (c->rf_cap < 2 * (size_t)khm) {
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "diag_hd refine sync");
            if (c->rf_buf) cudaFree(c->rf_buf);
            c->rf_buf = nullptr;
            c->rf_cap = 0;
            if ((e = cudaMalloc(&c->rf_buf, sizeof(double) * 2 * (size_t)khm)) != cudaSuccess)
                return cuda_fail(e, "diag_hd refine buffer");
            c->rf_cap = 2 * (size_t)khm;
        }
        if (oz_ws && (e = cudaMemsetAsync(d_rflag + 1, 0, sizeof(int), s)) != cudaSuccess)
            return cuda_fail(e, "diag_hd refine flag");
        stage_begin(c, 8);
        int rr = refine_apply(khm, Fsym, A, khm, eval, Fsym + (size_t)khm * khm, c->rf_buf, c->rf_buf + khm,
                              d_rflag, s, oz_ws, oz_bytes, oz_ws ? d_rflag + 1 : nullptr);
        stage_end(c, 8, 3);
        if (rr == BSRG_OK && oz_ws) {
            // the digit product reports a wait that ran out (1) or a non-finite input (2)
            int hf = 0;
            if ((e = cudaMemcpyAsync(&hf, d_rflag + 1, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess)
                return cuda_fail(e, "diag_hd refine flag");
            if (hf == 2) { set_error("diag_hd: non-finite value in the refinement product"); return BSRG_ERR_ARG; }
            if (hf) { set_error("diag_hd: a tensor-core wait timed out"); return BSRG_ERR_CUDA; }
        }
        // A V, the residuals and their sums, and the banded products of the Rayleigh-Ritz windows
        c->stage_flops[8] += 2.0 * (double)khm * khm * khm + 6.0 * (double)khm * khm + 132.0 * (double)khm * khm;
        if (rr != BSRG_OK) return rr;
        c->rf_n = khm;
    }
    if (gen && want_vectors) {
        // ---- x = L^-T y (diag_hd.f90:322-334, DTRSM('Left','L','T')) ----
        stage_begin(c, 6);
        int nl = 0;
        double *ctmp = chol_ws + (chol_workspace_doubles(khm_max) - (size_t)khm_max * 128 - 64);
        int rg = trsm_lower_left(khm, khm, Cov, khm, chol_ws, A, khm, true, ctmp, (size_t)khm_max * 128 + 64, s, &nl);
        stage_end(c, 6, nl);
        c->stage_flops[6] += (double)khm * khm * khm;
        if (rg != BSRG_OK) return rg;
    }
    if (bbout && (e = cudaMemcpyAsync(bbout, BB, sizeof(double) * nn * nch, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return cuda_fail(e, "diag_hd bb copy");
    if ((e = cudaMemcpyAsync(hi + o_fin, d_info + nch, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "diag_hd info");
    if (gen && (e = cudaMemcpyAsync(hi + o_fin + 1, d_cinfo, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "diag_hd info");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "diag_hd syevd");
    if (gen && hi[o_fin + 1] != 0) {
        set_error("BSR_HD: Cholesky factorization failed (overlap pivot %d)", hi[o_fin + 1]);
        return BSRG_ERR_INFO;
    }
    int hinfo = hi[o_fin];
    if (hinfo != 0) {
        set_error("LAP_DSYEV: DSYEV(lapack) gives INFO = %d", hinfo);
        return BSRG_ERR_INFO;
    }
    return stage_collect(c);
}

extern "C" int bsrg_diag_hd(bsrg_ctx *c, const bsrg_basis *b, int nch, const int *lch, const double *hcc,
                            int itype, int ilzero, int ibzero, double edmax, double egap, int want_vectors,
                            double *eval, int *khm_out, double *vecs, double *bbout)
{
    return diag_hd_impl(c, b, nch, lch, hcc, nullptr, itype, ilzero, ibzero, edmax, egap, want_vectors, eval,
                        khm_out, vecs, bbout);
}

extern "C" int bsrg_diag_hd_gen(bsrg_ctx *c, const bsrg_basis *b, int nch, const int *lch, const double *hcc,
                                const double *scc, int itype, int ilzero, int ibzero, double edmax, double egap,
                                int want_vectors, double *eval, int *khm_out, double *vecs, double *bbout)
{
    if (!scc) { set_error("diag_hd_gen: null overlap"); return BSRG_ERR_ARG; }
    return diag_hd_impl(c, b, nch, lch, hcc, scc, itype, ilzero, ibzero, edmax, egap, want_vectors, eval,
                        khm_out, vecs, bbout);
}

extern "C" int bsrg_ctx_set_refine(bsrg_ctx *c, int on)
{
    if (!c) { set_error("ctx_set_refine: null context"); return BSRG_ERR_ARG; }
    c->refine = on ? 1 : 0;
    return BSRG_OK;
}

extern "C" int bsrg_ctx_set_eigensolver(bsrg_ctx *c, int which)
{
    if (!c) { set_error("ctx_set_eigensolver: null context"); return BSRG_ERR_ARG; }
    if (which < 0 || which > 2) { set_error("ctx_set_eigensolver: which=%d (0, 1 or 2)", which); return BSRG_ERR_ARG; }
    c->eig_mode = which;
    return BSRG_OK;
}

extern "C" int bsrg_ctx_channel_fallbacks(const bsrg_ctx *c, int *count)
{
    if (!c || !count) { set_error("ctx_channel_fallbacks: null argument"); return BSRG_ERR_ARG; }
    *count = c->chan_fallbacks;
    return BSRG_OK;
}

extern "C" int bsrg_diag_hd_refine_stats(bsrg_ctx *c, int n, double *corr, double *resid)
{
    if (!c) { set_error("diag_hd_refine_stats: null context"); return BSRG_ERR_ARG; }
    if (n < 0 || n > c->rf_n) {
        set_error("diag_hd_refine_stats: n=%d but the last refined diag_hd had %d pairs", n, c->rf_n);
        return BSRG_ERR_ARG;
    }
    cudaError_t e;
    if (corr && n > 0 &&
        (e = cudaMemcpyAsync(corr, c->rf_buf, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess)
        return cuda_fail(e, "diag_hd_refine_stats");
    if (resid && n > 0 &&
        (e = cudaMemcpyAsync(resid, c->rf_buf + c->rf_n, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream)) !=
            cudaSuccess)
        return cuda_fail(e, "diag_hd_refine_stats");
    return BSRG_OK;
}

// whole path with host buffers: bsr_mat SUB1 followed by bsr_hd's diag_hd
extern "C" int bsrg_partial_wave_solve(bsrg_ctx *c, int ks, int ns, const double *t, double z, int nch,
                                       const int *lch, const double *ech, int norb, const double *P, int kmax,
                                       int ncoef, const int *ck, const int *ctype, const int *cich,
                                       const int *cjch, const int *ca, const int *cb, const double *cval,
                                       int want_vectors, double *eval, int *khm)
{
    if (!c || !t || !P || !eval || !khm) { set_error("partial_wave_solve: null argument"); return BSRG_ERR_ARG; }
    cudaStream_t s = c->stream;
    // the basis is the module state of define_spline: partial waves on one knot grid share
    // it, so it stays in the context until ks or a knot changes
    int rc = BSRG_OK;
    const bool same = c->pw_basis && c->pw_ks == ks && c->pw_knots->size() == (size_t)(ns + ks) &&
                      std::memcmp(c->pw_knots->data(), t, sizeof(double) * (ns + ks)) == 0;
    if (!same) {
        cudaStreamSynchronize(s);
        bsrg_basis_free(c->pw_basis);
        c->pw_basis = nullptr;
        c->pw_knots->clear();
        if ((rc = bsrg_define_spline(ks, ns, t, 0, 0, 0.0, s, &c->pw_basis)) != BSRG_OK) return rc;
        c->pw_knots->assign(t, t + ns + ks);
        c->pw_ks = ks;
    }
    const bsrg_basis *b = c->pw_basis;
    size_t nn = (size_t)ns * ns, nblk = (size_t)nch * (nch + 1) / 2;
    const size_t nh = (size_t)nch * ns;
    // device buffers live in the context between calls (grown when a larger wave arrives)
    size_t need = 0;
    auto add = [&](size_t bytes) { need += (bytes + 255) & ~(size_t)255; };
    add(sizeof(double) * ns * norb);
    add(sizeof(double) * nn * nblk);
    add(sizeof(double) * nh);
    if (want_vectors) add(sizeof(double) * nh * nh);
    cudaError_t e;
    if (c->pw_bytes < need) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) rc = cuda_fail(e, "partial_wave_solve sync");
        if (c->pw_buf) cudaFree(c->pw_buf);
        c->pw_buf = nullptr;
        c->pw_bytes = 0;
        if (rc == BSRG_OK && (e = cudaMalloc(&c->pw_buf, need)) != cudaSuccess)
            rc = cuda_fail(e, "partial_wave_solve alloc");
        if (rc == BSRG_OK) c->pw_bytes = need;
    }
    if (rc != BSRG_OK) return rc;
    Arena ar{(char *)c->pw_buf, 0, c->pw_bytes};
    double *dP = ar.take<double>((size_t)ns * norb), *hcc = ar.take<double>(nn * nblk);
    double *dev_eval = ar.take<double>(nh);
    double *vecs = want_vectors ? ar.take<double>(nh * nh) : nullptr;
    if ((e = cudaMemcpyAsync(dP, P, sizeof(double) * ns * norb, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        rc = cuda_fail(e, "partial_wave_solve upload");
    if (rc == BSRG_OK)
        rc = bsrg_assemble(c, b, z, nch, lch, ech, norb, dP, kmax, ncoef, ck, ctype, cich, cjch, ca, cb, cval, hcc,
                           nullptr, nullptr);
    if (rc == BSRG_OK)
        rc = bsrg_diag_hd(c, b, nch, lch, hcc, 0, 1, 1, 0.0, 0.001, want_vectors, dev_eval, khm, vecs, nullptr);
    if (rc == BSRG_OK &&
        (e = cudaMemcpyAsync(eval, dev_eval, sizeof(double) * (*khm), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        rc = cuda_fail(e, "partial_wave_solve download");
    if (rc == BSRG_OK && (e = cudaStreamSynchronize(s)) != cudaSuccess) rc = cuda_fail(e, "partial_wave_solve sync");
    cudaStreamSynchronize(s);
    return rc;
}
