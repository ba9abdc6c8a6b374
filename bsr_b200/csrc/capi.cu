// C ABI entry points (include/bsr_b200.h): argument checks, error reporting,
// basis lifecycle and the thin wrappers around the table and convolution
// kernels.  The assembly and eigensolve entry points live in assemble.cu and
// diag_hd.cu.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "bsrg_internal.h"

namespace bsrg {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *where)
{
    if (e == cudaSuccess) return BSRG_OK;
    set_error("%s: %s", where, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? BSRG_ERR_NOMEM : BSRG_ERR_CUDA;
}

cudaError_t smem_attr_raw(const void *func, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int &cur = limit[{dev, func}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// Gauss-Legendre rule on [0,1] by Newton iteration on the Legendre polynomial
// (the reference tabulates the same nodes to 15 digits, gauss.f90:2).
void gauss_legendre(int k, double *x, double *w)
{
    for (int i = 0; i < k; i++) {
        double z = std::cos(M_PI * (i + 0.75) / (k + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 200; it++) {
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= k; j++) {
                double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            dp = k * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) <= 1e-17) break;
        }
        double p0 = 1.0, p1 = z;
        for (int j = 2; j <= k; j++) {
            double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        if (k == 1) { p1 = z; p0 = 1.0; }
        dp = k * (z * p1 - p0) / (z * z - 1.0);
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
}

}  // namespace bsrg

using namespace bsrg;

#define CHECK_ARG(cond, ...)              \
    do {                                  \
        if (!(cond)) {                    \
            set_error(__VA_ARGS__);       \
            return BSRG_ERR_ARG;          \
        }                                 \
    } while (0)

extern "C" {

const char *bsrg_last_error(void) { return bsrg::g_err; }
int bsrg_version(void) { return 1; }

// define_grid.f90:86 (grid_type 0) and :213 (grid_type 1)
int bsrg_mkgrid(int grid_type, int ks, double z, double h, double hmax, double rmax, double *t, int cap,
                int *ns_out, int *ml_out, int *me_out, double *h_out)
{
    CHECK_ARG(t && ns_out && ml_out && me_out && h_out, "mkgrid: null output");
    CHECK_ARG(ks >= 2 && ks <= BSRG_MAXKS, "mkgrid: ks=%d out of range", ks);
    CHECK_ARG(z > 0 && h > 0 && hmax > 0 && rmax > 0, "mkgrid: non-positive parameter");
    if (grid_type == 0) {
        double h0 = h;
        int ml = (int)(1.0 / h + 0.1);
        CHECK_ARG(ml >= 1, "mkgrid: h too large");
        h = 1.0 / ml;
        double hp1 = 1.0 + h, tmax = z * rmax, hmx = z * hmax;
        double a = std::log(hmx / h) / std::log(hp1) + 1.0;
        int me1 = (int)(a > 0.0 ? a : 0.0);
        int me2 = (int)(std::log(tmax) / std::log(hp1) + 1.0);
        int me, m;
        double h2 = 0.0;
        if (me2 <= me1) { me = me2; m = 0; }
        else {
            me = me1;
            double tx = 1.0;
            for (int i = 0; i < me; i++) tx *= hp1;
            h2 = h * tx / hp1;
            m = (int)std::lround((tmax - tx) / h2);
        }
        int n = ml + me + m + ks - 1, nt = n + ks;
        CHECK_ARG(nt <= cap, "mkgrid: capacity %d < %d", cap, nt);
        for (int i = 0; i < nt; i++) t[i] = 0.0;
        for (int i = ks + 1; i <= ks + ml; i++) t[i - 1] = t[i - 2] + h0;
        for (int i = ks + ml + 1; i <= ks + me + ml; i++) t[i - 1] = t[i - 2] * hp1;
        for (int i = ks + me + ml + 1; i <= n + 1; i++) t[i - 1] = t[i - 2] + h2;
        for (int i = n + 2; i <= nt; i++) t[i - 1] = t[n];
        for (int i = 0; i < nt; i++) t[i] = t[i] / z;
        *ns_out = n; *ml_out = ml; *me_out = me; *h_out = h;
        return BSRG_OK;
    }
    CHECK_ARG(grid_type == 1, "mkgrid: unknown grid_type %d", grid_type);
    rmax = rmax * z;
    hmax = hmax * z;
    int nt = (int)((rmax / h + 1 + ks) * 2);
    CHECK_ARG(nt + ks <= cap, "mkgrid: capacity %d < %d", cap, nt + ks);
    std::vector<double> tt(nt + ks + 2, 0.0);
#define T1(i) tt[(i) - 1]
    int ns = ks;
    int ml = (int)(1.0 / h + 0.5);
    h = 1.0 / ml;
    for (int i = 1; i <= ml; i++) { ns++; T1(ns) = T1(ns - 1) + h; }
    if (hmax < h) hmax = h;
    int me = 0;
    for (;;) {
        CHECK_ARG(ns + 1 < nt, "mkgrid: grid overflow");
        T1(ns + 1) = T1(ns) * (1.0 + h);
        if (T1(ns + 1) - T1(ns) > hmax) break;
        ns++;
        if (T1(ns) > rmax) break;
        me++;
    }
    if (T1(ns) < rmax) {
        for (;;) {
            CHECK_ARG(ns + 1 < nt, "mkgrid: grid overflow");
            T1(ns + 1) = T1(ns) + hmax;
            ns++;
            if (T1(ns) >= rmax) break;
        }
    }
    if (T1(ns) > rmax) {
        ns--; me--;
        for (int i = ns + 1; i <= ns + ks; i++) T1(i) = rmax;
        T1(ns) = (T1(ns + 1) + T1(ns - 1)) / 2.0;
    }
#undef T1
    CHECK_ARG(ns + ks <= cap, "mkgrid: capacity %d < %d", cap, ns + ks);
    for (int i = 0; i < ns + ks; i++) t[i] = tt[i] / z;
    *ns_out = ns; *ml_out = ml; *me_out = me; *h_out = h;
    return BSRG_OK;
}

int bsrg_define_spline(int ks, int ns, const double *t_host, int ml, int me, double h, void *stream,
                       bsrg_basis **out)
{
    CHECK_ARG(out && t_host, "define_spline: null argument");
    CHECK_ARG(ks >= 2 && ks <= BSRG_MAXKS, "define_spline: ks=%d out of range 2..%d", ks, BSRG_MAXKS);
    CHECK_ARG(ns >= ks, "define_spline: ns=%d < ks=%d", ns, ks);
    for (int i = 1; i < ns + ks; i++)
        CHECK_ARG(t_host[i] >= t_host[i - 1], "define_spline: knots not non-decreasing at %d", i);
    for (int iv = 0; iv < ns - ks + 1; iv++)
        CHECK_ARG(t_host[iv + ks] > t_host[iv + ks - 1], "define_spline: empty interval %d", iv);
    cudaStream_t s = (cudaStream_t)stream;
    bsrg_basis *b = new bsrg_basis();
    std::memset(b, 0, sizeof *b);
    b->ks = ks; b->ns = ns; b->nv = ns - ks + 1; b->ml = ml; b->me = me; b->h = h;
    cudaGetDevice(&b->device);
    gauss_legendre(ks, b->gx, b->gw);
    size_t nvk = (size_t)b->nv * ks, nb = (size_t)(b->nv + 1) * ks * ks, nband = (size_t)ns * ks;
    double **bufs[] = {&b->t, &b->gr, &b->grm, &b->grw, &b->bsp, &b->bsq, &b->bspd,
                       &b->sb, &b->r1, &b->rm1, &b->rm2, &b->rm3, &b->db1, &b->db2};
    size_t sizes[] = {(size_t)(ns + ks), nvk, nvk, nvk, nb, nb, 2 * nb,
                      nband, nband, nband, nband, nband, nband, nband};
    for (int q = 0; q < 14; q++) {
        cudaError_t e = cudaMalloc((void **)bufs[q], sizes[q] * sizeof(double));
        if (e != cudaSuccess) { bsrg_basis_free(b); return cuda_fail(e, "define_spline alloc"); }
        // allocate_grid / allocate_galerkin zero the module arrays (spline_grid.f90:49)
        e = cudaMemsetAsync(*bufs[q], 0, sizes[q] * sizeof(double), (cudaStream_t)stream);
        if (e != cudaSuccess) { bsrg_basis_free(b); return cuda_fail(e, "define_spline zero"); }
    }
    cudaError_t e = cudaMemcpyAsync(b->t, t_host, sizeof(double) * (ns + ks), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { bsrg_basis_free(b); return cuda_fail(e, "define_spline copy"); }
    int rc = launch_basis_tables(b, s);
    if (rc != BSRG_OK) { bsrg_basis_free(b); return rc; }
    *out = b;
    return BSRG_OK;
}

int bsrg_basis_free(bsrg_basis *b)
{
    if (!b) return BSRG_OK;
    double *bufs[] = {b->t, b->gr, b->grm, b->grw, b->bsp, b->bsq, b->bspd,
                      b->sb, b->r1, b->rm1, b->rm2, b->rm3, b->db1, b->db2};
    for (double *p : bufs)
        if (p) cudaFree(p);
    delete b;
    return BSRG_OK;
}

int bsrg_basis_dims(const bsrg_basis *b, int *dims)
{
    CHECK_ARG(b && dims, "basis_dims: null argument");
    dims[0] = b->ks; dims[1] = b->ns; dims[2] = b->nv; dims[3] = b->ml; dims[4] = b->me;
    return BSRG_OK;
}

}  // extern "C"

namespace bsrg {
// Full_mat_sym(ns, ks, sb, bb, 'l') (full_mat.f90): the full symmetric ns x ns matrix of the band
__global__ void full_from_band_sym_kernel(int ns, int ks, const double *__restrict__ sb, double *bb)
{
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)ns * ns) return;
    const int i = (int)(idx % ns), j = (int)(idx / ns);
    const int hi = i > j ? i : j, lo = i > j ? j : i;
    bb[idx] = hi - lo < ks ? sb[hi + (size_t)ns * (lo - hi + ks - 1)] : 0.0;
}

// facsb (facsb.f90:2-36): bs = sb^T in upper band storage (ks, ns) with the r = 0 boundary
// condition (first row and column replaced by e_1), then its banded Cholesky factor U
// (DPBTRF('U', ns, ks-1, bs, ks): bs(ks+i-j, j) = U(i, j)), left-looking, one thread.
__global__ void facsb_kernel(int ns, int ks, const double *__restrict__ sb, double *bs, int *info)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int kd = ks - 1;
    for (int j = 0; j < ns; j++)
        for (int m = 0; m < ks; m++) bs[m + (size_t)ks * j] = sb[j + (size_t)ns * m];
    for (int m = 0; m < ks - 1; m++) bs[m + (size_t)ks * (ks - 1 - m)] = 0.0;
    bs[(ks - 1)] = 1.0;
    auto U = [&](int i, int j) -> double & { return bs[(kd + i - j) + (size_t)ks * j]; };   // 0-based i <= j
    *info = 0;
    for (int j = 0; j < ns; j++) {
        const int k0 = j - kd > 0 ? j - kd : 0;
        for (int i = k0; i < j; i++) {
            double s = U(i, j);
            for (int k = k0; k < i; k++) s -= U(k, i) * U(k, j);
            U(i, j) = s / U(i, i);
        }
        double d = U(j, j);
        for (int k = k0; k < j; k++) d -= U(k, j) * U(k, j);
        if (!(d > 0.0)) { *info = j + 1; return; }
        U(j, j) = sqrt(d);
    }
}
}  // namespace bsrg

extern "C" {

int bsrg_basis_get(const bsrg_basis *b, int which, double *dst, void *stream)
{
    if (b && dst && (which == 14 || which == 15)) {
        cudaStream_t s = (cudaStream_t)stream;
        if (which == 14) {
            const long nn = (long)b->ns * b->ns;
            full_from_band_sym_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(b->ns, b->ks, b->sb, dst);
            return cuda_fail(cudaGetLastError(), "basis_get bb");
        }
        int *dinfo = nullptr;
        cudaError_t e = cudaMallocAsync((void **)&dinfo, sizeof(int), s);
        if (e != cudaSuccess) return cuda_fail(e, "basis_get bs");
        facsb_kernel<<<1, 32, 0, s>>>(b->ns, b->ks, b->sb, dst, dinfo);
        int hinfo = 0;
        e = cudaMemcpyAsync(&hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFreeAsync(dinfo, s);
        if (e != cudaSuccess) return cuda_fail(e, "basis_get bs");
        if (hinfo != 0) { set_error("facsb: dpbtrf (LAPACK) failed (column %d)", hinfo); return BSRG_ERR_INFO; }
        return BSRG_OK;
    }
    CHECK_ARG(b && dst, "basis_get: null argument");
    size_t nvk = (size_t)b->nv * b->ks, nb = (size_t)(b->nv + 1) * b->ks * b->ks,
           nband = (size_t)b->ns * b->ks;
    const double *src;
    size_t n;
    switch (which) {
    case 0: src = b->gr; n = nvk; break;
    case 1: src = b->grm; n = nvk; break;
    case 2: src = b->grw; n = nvk; break;
    case 3: src = b->bsp; n = nb; break;
    case 4: src = b->bsq; n = nb; break;
    case 5: src = b->bspd; n = 2 * nb; break;
    case 6: src = b->sb; n = nband; break;
    case 7: src = b->r1; n = nband; break;
    case 8: src = b->rm1; n = nband; break;
    case 9: src = b->rm2; n = nband; break;
    case 10: src = b->rm3; n = nband; break;
    case 11: src = b->db1; n = nband; break;
    case 12: src = b->db2; n = nband; break;
    case 13: src = b->t; n = (size_t)(b->ns + b->ks); break;
    default: set_error("basis_get: unknown array %d", which); return BSRG_ERR_ARG;
    }
    return cuda_fail(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                     (cudaStream_t)stream), "basis_get");
}

int bsrg_mrm(const bsrg_basis *b, int mm, double *rm, void *stream)
{
    CHECK_ARG(b && rm, "mrm: null argument");
    return launch_mrm(b, mm, rm, (cudaStream_t)stream);
}

int bsrg_rk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream)
{
    CHECK_ARG(b, "rk_moments: null basis");
    CHECK_ARG(k >= 0 && k <= 64, "rk_moments: k=%d out of range", k);
    return launch_rk_moments(b, k, rkd1, rkd2, rkd, (cudaStream_t)stream);
}

int bsrg_mrk_cell_from_moments(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd,
                               double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkd1 && rkd2 && rkd && rkb, "mrk_cell: null argument");
    CHECK_ARG(ldp >= b->ks, "mrk_cell: ldp=%d < ks=%d", ldp, b->ks);
    return launch_mrk_cell(b, rkd1, rkd2, rkd, rkb, ldp, (cudaStream_t)stream);
}

int bsrg_mrk_cell(const bsrg_basis *b, int k, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mrk_cell: null argument");
    CHECK_ARG(ldp >= b->ks, "mrk_cell: ldp=%d < ks=%d", ldp, b->ks);
    CHECK_ARG(k >= 0 && k <= 64, "mrk_cell: k=%d out of range", k);
    cudaStream_t s = (cudaStream_t)stream;
    int ik = ik_of(b->ks);
    size_t n1 = (size_t)ik * b->nv, n3 = (size_t)ik * ik * b->nv;
    double *buf = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&buf, (2 * n1 + n3) * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "mrk_cell scratch");
    int rc = launch_rk_moments(b, k, buf, buf + n1, buf + 2 * n1, s);
    if (rc == BSRG_OK) rc = launch_mrk_cell(b, buf, buf + n1, buf + 2 * n1, rkb, ldp, s);
    cudaFreeAsync(buf, s);
    return rc;
}

int bsrg_nk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream)
{
    CHECK_ARG(b, "nk_moments: null basis");
    CHECK_ARG(k >= -1 && k <= 64, "nk_moments: k=%d out of range", k);
    return launch_nkmk_moments(b, k, 0, rkd1, rkd2, rkd, (cudaStream_t)stream);
}

int bsrg_mk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream)
{
    CHECK_ARG(b, "mk_moments: null basis");
    CHECK_ARG(k >= -1 && k <= 64, "mk_moments: k=%d out of range", k);
    return launch_nkmk_moments(b, k, 1, rkd1, rkd2, rkd, (cudaStream_t)stream);
}

int bsrg_mmk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mmk_cell: null argument");
    CHECK_ARG(ldp >= b->ks, "mmk_cell: ldp=%d < ks=%d", ldp, b->ks);
    CHECK_ARG(k >= -1 && k <= 64, "mmk_cell: k=%d out of range", k);
    cudaStream_t s = (cudaStream_t)stream;
    int ik = ik_of(b->ks);
    size_t n1 = (size_t)ik * b->nv, n3 = (size_t)ik * ik * b->nv;
    double *buf = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&buf, (2 * n1 + n3) * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "mmk_cell scratch");
    int rc = launch_nkmk_moments(b, k, 1, buf, buf + n1, buf + 2 * n1, s);
    if (rc == BSRG_OK) rc = launch_mrk_cell_scaled(b, buf, buf + n1, buf + 2 * n1, fine, rkb, ldp, s);
    cudaFreeAsync(buf, s);
    return rc;
}

int bsrg_mnk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mnk_cell: null argument");
    CHECK_ARG(ldp >= b->ks, "mnk_cell: ldp=%d < ks=%d", ldp, b->ks);
    CHECK_ARG(k >= -1 && k <= 64, "mnk_cell: k=%d out of range", k);
    cudaStream_t s = (cudaStream_t)stream;
    int ik = ik_of(b->ks);
    size_t n1 = (size_t)ik * b->nv, n3 = (size_t)ik * ik * b->nv;
    double *buf = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&buf, (2 * n1 + n3) * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "mnk_cell scratch");
    int rc = launch_nkmk_moments(b, k, 0, buf, buf + n1, buf + 2 * n1, s);
    if (rc == BSRG_OK) rc = launch_mnk_cell(b, buf, buf + n1, buf + 2 * n1, fine, rkb, ldp, s);
    cudaFreeAsync(buf, s);
    return rc;
}

int bsrg_tk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream)
{
    CHECK_ARG(b, "tk_moments: null basis");
    CHECK_ARG(k >= 0 && k <= 64, "tk_moments: k=%d out of range", k);
    return launch_tk_moments(b, k, rkd1, rkd2, rkd, (cudaStream_t)stream);
}

int bsrg_mtk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mtk_cell: null argument");
    CHECK_ARG(ldp >= 2 * b->ks - 1, "mtk_cell: ldp=%d < 2ks-1=%d", ldp, 2 * b->ks - 1);
    CHECK_ARG(k >= 0 && k <= 64, "mtk_cell: k=%d out of range", k);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t jk = (size_t)b->ks * b->ks, n1 = jk * b->nv, n3 = jk * jk * b->nv;
    double *buf = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&buf, (2 * n1 + n3) * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "mtk_cell scratch");
    int rc = launch_tk_moments(b, k, buf, buf + n1, buf + 2 * n1, s);
    if (rc == BSRG_OK) rc = launch_mtk_cell(b, k, buf, buf + n1, buf + 2 * n1, fine, rkb, ldp, s);
    cudaFreeAsync(buf, s);
    return rc;
}

// V^k (mode 0) and W^k (mode 1) share the layouts; W^k's moment combinations need a
// ks*ks*nv scratch, which bsrg_wk_moments allocates and frees
static int vw_moments_call(const bsrg_basis *b, int k, int mode, double *rkd1, double *rkd2, double *rkd3,
                           double *rkd4, double *rkd, cudaStream_t s)
{
    double *tmp = nullptr;
    if (mode && (rkd3 || rkd4)) {
        cudaError_t e = cudaMallocAsync((void **)&tmp, sizeof(double) * (size_t)b->ks * b->ks * b->nv, s);
        if (e != cudaSuccess) return cuda_fail(e, "wk_moments scratch");
    }
    int rc = launch_vw_moments(b, k, mode, rkd1, rkd2, rkd3, rkd4, rkd, tmp, s);
    if (tmp) cudaFreeAsync(tmp, s);
    return rc;
}

int bsrg_vk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd,
                    void *stream)
{
    CHECK_ARG(b, "vk_moments: null basis");
    CHECK_ARG(k >= 0 && k <= 64, "vk_moments: k=%d out of range", k);
    return vw_moments_call(b, k, 0, rkd1, rkd2, rkd3, rkd4, rkd, (cudaStream_t)stream);
}

int bsrg_wk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd,
                    void *stream)
{
    CHECK_ARG(b, "wk_moments: null basis");
    CHECK_ARG(k >= 0 && k <= 64, "wk_moments: k=%d out of range", k);
    return vw_moments_call(b, k, 1, rkd1, rkd2, rkd3, rkd4, rkd, (cudaStream_t)stream);
}

static int mvw_cell_call(const bsrg_basis *b, int k, int mode, double fine, double *rkb, int ldp, cudaStream_t s)
{
    const size_t jk = (size_t)b->ks * b->ks, nv = (size_t)b->nv;
    const size_t nj = mode == 2 ? jk : (size_t)ik_of(b->ks);       // pairs on the r2 side
    double *buf = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&buf, (2 * nj * nv + 3 * jk * nv + jk * nj * nv) * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "m?k_cell scratch");
    double *r1 = buf, *r2 = r1 + nj * nv, *r3 = r2 + nj * nv, *r4 = r3 + jk * nv, *rd = r4 + jk * nv;
    double *tmp = rd + jk * nj * nv;
    int rc = launch_vw_moments(b, k, mode, r1, r2, r3, r4, rd, tmp, s);
    if (rc == BSRG_OK)
        rc = mode == 2 ? launch_mqk_cell(b, r1, r2, r3, r4, rd, fine, rkb, ldp, s)
                       : launch_mvk_cell(b, r1, r2, r3, r4, rd, fine, rkb, ldp, s);
    cudaFreeAsync(buf, s);
    return rc;
}

int bsrg_mvk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mvk_cell: null argument");
    CHECK_ARG(ldp >= 2 * b->ks - 1, "mvk_cell: ldp=%d < 2ks-1=%d", ldp, 2 * b->ks - 1);
    CHECK_ARG(k >= 0 && k <= 64, "mvk_cell: k=%d out of range", k);
    return mvw_cell_call(b, k, 0, fine, rkb, ldp, (cudaStream_t)stream);
}

int bsrg_qk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd,
                    void *stream)
{
    CHECK_ARG(b, "qk_moments: null basis");
    CHECK_ARG(k >= 0 && k <= 64, "qk_moments: k=%d out of range", k);
    return vw_moments_call(b, k, 2, rkd1, rkd2, rkd3, rkd4, rkd, (cudaStream_t)stream);
}

int bsrg_mqk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mqk_cell: null argument");
    CHECK_ARG(ldp >= 2 * b->ks - 1, "mqk_cell: ldp=%d < 2ks-1=%d", ldp, 2 * b->ks - 1);
    CHECK_ARG(k >= 0 && k <= 64, "mqk_cell: k=%d out of range", k);
    return mvw_cell_call(b, k, 2, fine, rkb, ldp, (cudaStream_t)stream);
}

int bsrg_mwk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream)
{
    CHECK_ARG(b && rkb, "mwk_cell: null argument");
    CHECK_ARG(ldp >= 2 * b->ks - 1, "mwk_cell: ldp=%d < 2ks-1=%d", ldp, 2 * b->ks - 1);
    CHECK_ARG(k >= 0 && k <= 64, "mwk_cell: k=%d out of range", k);
    return mvw_cell_call(b, k, 1, fine, rkb, ldp, (cudaStream_t)stream);
}

int bsrg_density(int ns, int ks, double *d, const double *p1, const double *p2, char type, void *stream)
{
    CHECK_ARG(d && p1 && p2, "density: null argument");
    CHECK_ARG(ns >= ks && ks >= 1, "density: bad ns/ks");
    CHECK_ARG(type == 's' || type == 'n' || type == 'x', "density: unknown type '%c'", type);
    return launch_density(ns, ks, d, p1, p2, type, (cudaStream_t)stream);
}

int bsrg_convol(int ns, int ks, double *a, const double *d, const double *rkb, int ldp, int icase, char sym_i,
                char sym_j, void *stream)
{
    CHECK_ARG(a && d && rkb, "convol: null argument");
    CHECK_ARG(ns >= ks && ks >= 1, "convol: bad ns/ks");
    if (!((sym_i == 's' || sym_i == 'n') && (sym_j == 's' || sym_j == 'n') && icase >= 1 && icase <= 4)) {
        set_error(" CONVOL:  unknown case (icase=%d sym_i=%c sym_j=%c)", icase, sym_i, sym_j);
        return BSRG_ERR_CASE;
    }
    int need = (sym_i == 'n' || sym_j == 'n') ? 2 * ks - 1 : ks;
    CHECK_ARG(ldp >= need, "convol: ldp=%d < %d", ldp, need);
    return launch_convol(ns, ks, a, d, rkb, ldp, icase, sym_i, sym_j, (cudaStream_t)stream);
}

int bsrg_bav(int ns, int ks, const double *b, const double *v, double *y, char type, char side, void *stream)
{
    CHECK_ARG(b && v && y, "bav: null argument");
    CHECK_ARG(type == 's' || (type == 'n' && (side == 'r' || side == 'l')), "bav: type '%c' side '%c'", type, side);
    return launch_bav(ns, ks, b, v, y, type, side, (cudaStream_t)stream);
}

int bsrg_bvmv(int n, int k, const double *ar, char type, const double *x, const double *y, double *out,
              void *stream)
{
    CHECK_ARG(ar && x && y && out, "bvmv: null argument");
    CHECK_ARG(n >= 2 && k >= 2, "bvmv: n=%d k=%d", n, k);
    return launch_bvmv(n, k, ar, type, x, y, out, (cudaStream_t)stream);
}

int bsrg_quadr(const bsrg_basis *b, const double *p1, const double *p2, int m, double *out, void *stream)
{
    CHECK_ARG(b && p1 && p2 && out, "quadr: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const double *rm = m == 1 ? b->r1 : m == 0 ? b->sb : m == -1 ? b->rm1 : m == -2 ? b->rm2 : nullptr;
    double *tmp = nullptr;
    if (!rm) {
        cudaError_t e = cudaMallocAsync((void **)&tmp, sizeof(double) * (size_t)b->ns * b->ks, s);
        if (e != cudaSuccess) return cuda_fail(e, "quadr");
        int rc = launch_mrm(b, m, tmp, s);
        if (rc != BSRG_OK) { cudaFreeAsync(tmp, s); return rc; }
        rm = tmp;
    }
    int rc = launch_bvmv(b->ns, b->ks, rm, 's', p1, p2, out, s);
    if (tmp) cudaFreeAsync(tmp, s);
    return rc;
}

int bsrg_sum_amb(int ns, int ks, const double *a, const double *b, char sym, double *out, void *stream)
{
    CHECK_ARG(a && b && out, "sum_amb: null argument");
    if (!(sym == 's' || sym == 'l' || sym == 'n' || sym == 'x')) {
        set_error(" SUM_AmB:  unknown symmetry '%c'", sym);
        return BSRG_ERR_CASE;
    }
    return launch_sum_amb(ns, ks, a, b, sym, out, (cudaStream_t)stream);
}

}  // extern "C"
