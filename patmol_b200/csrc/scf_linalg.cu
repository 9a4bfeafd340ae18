// scf_linalg.cu -- the dense linear algebra of one SCF iteration on the
// GPU: the step of rhf_scf_update (rhfscf.c:36-47) after the Fock matrix is
// formed.  The reference does it on the host: spack_trans (X^T F X,
// spack_math.c:327-384), spack_diag (Householder + implicit QL,
// spack_math.c:300-320), form_cmatrix (C = X W, scfaux.c:5-21) and
// form_pmatrix (P = C_occ C_occ^T, scfaux.c:24-41).  Here the products are
// cuBLAS DGEMMs and the symmetric eigenproblem is cuSOLVER's divide and
// conquer (syevd); a context holds X and every work array, so an update
// allocates nothing.
//
// Layouts: X comes from the caller row-major n x nx (C order), i.e. the
// column-major nx x n matrix Xc = X^T.  With F symmetric:
//   T  = F Xc^T          (n x nx)      Fp = Xc T = X^T F X   (nx x nx)
//   Fp V = V diag(e)     (syevd, ascending e)
//   C  = Xc^T V = X V    (n x nx, column a = orbital a)
//   P  = C_occ C_occ^T,  W = C_occ diag(e_occ) C_occ^T      (n x n, packed on output)
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include "../../include/patgpu.h"

namespace pg {
int fail(int code, const char *fmt, ...);
}
using pg::fail;

struct patgpu_scf_s {
    int n = 0, nx = 0, nocc = 0;
    cublasHandle_t cb = nullptr;
    cusolverDnHandle_t cs = nullptr;
    double *X = nullptr, *F = nullptr, *T = nullptr, *Fp = nullptr, *e = nullptr, *C = nullptr, *Cs = nullptr,
           *Pf = nullptr, *work = nullptr;
    double *pkF = nullptr, *pkP = nullptr, *pkW = nullptr;   // packed staging of the host-buffer form
    cudaStream_t own = nullptr;
    int *info = nullptr;
    int lwork = 0;
};

namespace {

__global__ void unpack_sym_kernel(const double *__restrict__ pk, double *__restrict__ full, int n)
{
    const long long tot = (long long)n * n;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / n), j = (int)(idx % n);
        const int r = i > j ? i : j, c = i > j ? j : i;
        full[idx] = pk[(long long)r * (r + 1) / 2 + c];
    }
}

// packed lower triangle (row-major, ij = i(i+1)/2 + j) of a symmetric matrix
__global__ void pack_sym_kernel(const double *__restrict__ full, double *__restrict__ pk, int n)
{
    const long long no2 = (long long)n * (n + 1) / 2;
    for (long long ij = (long long)blockIdx.x * blockDim.x + threadIdx.x; ij < no2;
         ij += (long long)gridDim.x * blockDim.x) {
        int i = (int)((sqrt(8.0 * (double)ij + 1.0) - 1.0) * 0.5);
        while ((long long)(i + 1) * (i + 2) / 2 <= ij) ++i;
        while ((long long)i * (i + 1) / 2 > ij) --i;
        const int j = (int)(ij - (long long)i * (i + 1) / 2);
        pk[ij] = full[(size_t)j * n + i];
    }
}

// Cs[:, a] = e[a] C[:, a] for the occupied columns
__global__ void scale_cols_kernel(const double *__restrict__ C, const double *__restrict__ e, double *__restrict__ Cs,
                                  int n, int nocc)
{
    const long long tot = (long long)n * nocc;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
         idx += (long long)gridDim.x * blockDim.x)
        Cs[idx] = C[idx] * e[idx / n];
}

int grid(long long work) { return (int)((work + 255) / 256 < 4096 ? (work + 255) / 256 : 4096); }

}  // namespace

extern "C" {

int patgpu_scf_create(int n, int nx, int nocc, const double *X, patgpu_scf *out)
{
    if (!out || n < 1 || nx < 1 || nx > n || nocc < 1 || nocc > nx || !X)
        return fail(PATGPU_EINVAL, "patgpu_scf_create: bad argument");
    *out = nullptr;
    auto *s = new patgpu_scf_s();
    s->n = n;
    s->nx = nx;
    s->nocc = nocc;
    const size_t nn = (size_t)n * n, nxn = (size_t)n * nx;
    bool ok = cublasCreate(&s->cb) == CUBLAS_STATUS_SUCCESS && cusolverDnCreate(&s->cs) == CUSOLVER_STATUS_SUCCESS;
    ok = ok && cudaMalloc(&s->X, sizeof(double) * nxn) == cudaSuccess;
    ok = ok && cudaMalloc(&s->F, sizeof(double) * nn) == cudaSuccess;
    ok = ok && cudaMalloc(&s->T, sizeof(double) * nxn) == cudaSuccess;
    ok = ok && cudaMalloc(&s->Fp, sizeof(double) * (size_t)nx * nx) == cudaSuccess;
    ok = ok && cudaMalloc(&s->e, sizeof(double) * nx) == cudaSuccess;
    ok = ok && cudaMalloc(&s->C, sizeof(double) * nxn) == cudaSuccess;
    ok = ok && cudaMalloc(&s->Cs, sizeof(double) * (size_t)n * nocc) == cudaSuccess;
    ok = ok && cudaMalloc(&s->Pf, sizeof(double) * nn) == cudaSuccess;
    ok = ok && cudaMalloc(&s->info, sizeof(int)) == cudaSuccess;
    const size_t no2 = (size_t)n * (n + 1) / 2;
    ok = ok && cudaMalloc(&s->pkF, sizeof(double) * no2) == cudaSuccess;
    ok = ok && cudaMalloc(&s->pkP, sizeof(double) * no2) == cudaSuccess;
    ok = ok && cudaMalloc(&s->pkW, sizeof(double) * no2) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMemcpy(s->X, X, sizeof(double) * nxn, cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cusolverDnDsyevd_bufferSize(s->cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nx, s->Fp, nx,
                                           s->e, &s->lwork) == CUSOLVER_STATUS_SUCCESS;
    ok = ok && cudaMalloc(&s->work, sizeof(double) * (size_t)(s->lwork > 0 ? s->lwork : 1)) == cudaSuccess;
    if (!ok) {
        patgpu_scf_destroy(s);
        return fail(PATGPU_ECUDA, "patgpu_scf_create: cuBLAS/cuSOLVER set-up or device allocation failed");
    }
    *out = s;
    return 0;
}

int patgpu_scf_destroy(patgpu_scf s)
{
    if (!s) return 0;
    for (double *p : {s->X, s->F, s->T, s->Fp, s->e, s->C, s->Cs, s->Pf, s->work, s->pkF, s->pkP, s->pkW})
        if (p) cudaFree(p);
    if (s->own) cudaStreamDestroy(s->own);
    if (s->info) cudaFree(s->info);
    if (s->cb) cublasDestroy(s->cb);
    if (s->cs) cusolverDnDestroy(s->cs);
    delete s;
    return 0;
}

int patgpu_scf_density(patgpu_scf s, const double *dF, double *dP, double *dW, double *eps, double *C,
                       void *stream)
{
    if (!s || !dF || !dP) return fail(PATGPU_EINVAL, "patgpu_scf_density: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int n = s->n, nx = s->nx, no = s->nocc;
    const double one = 1.0, zero = 0.0;
    if (cublasSetStream(s->cb, st) != CUBLAS_STATUS_SUCCESS || cusolverDnSetStream(s->cs, st) != CUSOLVER_STATUS_SUCCESS)
        return fail(PATGPU_ECUDA, "patgpu_scf_density: stream");
    unpack_sym_kernel<<<grid((long long)n * n), 256, 0, st>>>(dF, s->F, n);
    bool ok = cudaGetLastError() == cudaSuccess;
    // T = F Xc^T ; Fp = Xc T
    ok = ok && cublasDgemm(s->cb, CUBLAS_OP_N, CUBLAS_OP_T, n, nx, n, &one, s->F, n, s->X, nx, &zero, s->T, n) ==
                   CUBLAS_STATUS_SUCCESS;
    ok = ok && cublasDgemm(s->cb, CUBLAS_OP_N, CUBLAS_OP_N, nx, nx, n, &one, s->X, nx, s->T, n, &zero, s->Fp, nx) ==
                   CUBLAS_STATUS_SUCCESS;
    ok = ok && cusolverDnDsyevd(s->cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nx, s->Fp, nx, s->e, s->work,
                                s->lwork, s->info) == CUSOLVER_STATUS_SUCCESS;
    // C = Xc^T V
    ok = ok && cublasDgemm(s->cb, CUBLAS_OP_T, CUBLAS_OP_N, n, nx, nx, &one, s->X, nx, s->Fp, nx, &zero, s->C, n) ==
                   CUBLAS_STATUS_SUCCESS;
    // P = C_occ C_occ^T
    ok = ok && cublasDgemm(s->cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, no, &one, s->C, n, s->C, n, &zero, s->Pf, n) ==
                   CUBLAS_STATUS_SUCCESS;
    if (!ok) return fail(PATGPU_ECUDA, "patgpu_scf_density: cuBLAS/cuSOLVER call failed");
    pack_sym_kernel<<<grid((long long)n * (n + 1) / 2), 256, 0, st>>>(s->Pf, dP, n);
    if (dW) {
        scale_cols_kernel<<<grid((long long)n * no), 256, 0, st>>>(s->C, s->e, s->Cs, n, no);
        ok = cublasDgemm(s->cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, no, &one, s->Cs, n, s->C, n, &zero, s->Pf, n) ==
             CUBLAS_STATUS_SUCCESS;
        if (!ok) return fail(PATGPU_ECUDA, "patgpu_scf_density: cuBLAS call failed");
        pack_sym_kernel<<<grid((long long)n * (n + 1) / 2), 256, 0, st>>>(s->Pf, dW, n);
    }
    int info = 0;
    if (cudaMemcpyAsync(&info, s->info, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return fail(PATGPU_ECUDA, "patgpu_scf_density: info copy");
    if (eps && cudaMemcpyAsync(eps, s->e, sizeof(double) * nx, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return fail(PATGPU_ECUDA, "patgpu_scf_density: eigenvalue copy");
    if (C && cudaMemcpyAsync(C, s->C, sizeof(double) * (size_t)n * nx, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return fail(PATGPU_ECUDA, "patgpu_scf_density: orbital copy");
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return fail(PATGPU_ECUDA, "patgpu_scf_density: %s", cudaGetErrorString(cudaGetLastError()));
    if (info != 0) return fail(PATGPU_ECUDA, "patgpu_scf_density: syevd info %d", info);
    return 0;
}

int patgpu_scf_density_host(patgpu_scf s, const double *F, double *P, double *W, double *eps, double *C)
{
    if (!s || !F || !P) return fail(PATGPU_EINVAL, "patgpu_scf_density_host: null argument");
    const size_t no2 = (size_t)s->n * (s->n + 1) / 2;
    if (cudaMemcpyAsync(s->pkF, F, sizeof(double) * no2, cudaMemcpyHostToDevice, s->own) != cudaSuccess)
        return fail(PATGPU_ECUDA, "patgpu_scf_density_host: copy in");
    int rc = patgpu_scf_density(s, s->pkF, s->pkP, W ? s->pkW : nullptr, eps, C, s->own);
    if (rc) return rc;
    bool ok = cudaMemcpyAsync(P, s->pkP, sizeof(double) * no2, cudaMemcpyDeviceToHost, s->own) == cudaSuccess;
    if (W) ok = ok && cudaMemcpyAsync(W, s->pkW, sizeof(double) * no2, cudaMemcpyDeviceToHost, s->own) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s->own) == cudaSuccess;
    return ok ? 0 : fail(PATGPU_ECUDA, "patgpu_scf_density_host: copy out");
}

}  // extern "C"
