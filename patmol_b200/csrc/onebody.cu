// onebody.cu -- one-body integrals by McMurchie-Davidson on the GPU.
//
// One thread per (shell pair, component pair) of the packed lower triangle.
// Per primitive pair: Hermite expansion coefficients E^{ij}_t per direction
// (the recursion of mdd.c:3-43), Hermite Coulomb integrals R_tuv from the
// Boys function (the quantities mdr.c:37-2163 tabulates, here by the
// recursion R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X R^{n+1}_{t,u,v}), then
//   S = c s12 E^x_0 E^y_0 E^z_0                              (oneints.c:80)
//   T = c s12 sum_d T_d prod_{d' != d} E^{d'}_0              (oneints.c:81-116)
//   V = c sum_C -q_C sum_tuv E_t E_u E_v R_tuv(p, P - C)     (oneints.c:48-72,117-127)
//   V_DPM = sum_g sum_tuv E_t E_u E_v R_tuv(w_g, P - Q) s_g  (dpmints.c:75-114)
// with the six model Gaussians of dpmints.c:30-36 at the positron centre Q.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/patgpu.h"
#include "common.cuh"
#include "onebody.cuh"

namespace pg {

__constant__ int c_cart1[4][10];
__constant__ double c_norm1[4][10];
// model charge of the distributed positron model (dpmints.c:30-36)
__constant__ double c_palf[6] = {6.8505018000, 4.0491646000, 3.5941062989,
                                 1.2478274000, 0.7927690989, 0.3377107978};
__constant__ double c_pcof[6] = {0.0766926784, 0.1483475912, 0.0462334641,
                                 0.0717376427, 0.0447149792, 0.0069678529};

cudaError_t upload_onebody_constants()
{
    int cart[4][10] = {};
    double nrm[4][10] = {};
    for (int l = 0; l <= 3; ++l)
        for (int k = 0; k < ncart(l); ++k) {
            cart[l][k] = kCart.e[l][k];
            nrm[l][k] = 1.0 / sqrt(dfact_odd(cart_x(l, k)) * dfact_odd(cart_y(l, k)) * dfact_odd(cart_z(l, k)));
        }
    cudaError_t e = cudaMemcpyToSymbol(c_cart1, cart, sizeof(cart));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_norm1, nrm, sizeof(nrm));
    return e;
}

struct OneArgs {
    const int *item;     // per thread: ish, jsh, ia, ib, packed index
    int nitem;
    const int *l, *cen, *poff;
    const double *al, *co, *q, *xyz;
    int ncen, skipcen;
    double *S, *T, *H, *V;   // packed outputs (V: DPM potential)
};

#define EM 5      // l + 1 + 1 for l <= 3
#define ET 10

// E[i][j][t] for i <= la, j <= lb (M > la, lb)
template <int M>
__device__ void herm_e(double E[M][M][ET], int la, int lb, double h, double pa, double pb)
{
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j <= lb; ++j)
            for (int t = 0; t <= la + lb; ++t) E[i][j][t] = 0.0;
    E[0][0][0] = 1.0;
    for (int j = 0; j < lb; ++j)
        for (int t = 0; t <= j + 1; ++t) {
            double v = (t <= j ? pb * E[0][j][t] : 0.0) + (t + 1 <= j ? (t + 1) * E[0][j][t + 1] : 0.0);
            if (t > 0) v += h * E[0][j][t - 1];
            E[0][j + 1][t] = v;
        }
    for (int i = 0; i < la; ++i)
        for (int j = 0; j <= lb; ++j)
            for (int t = 0; t <= i + j + 1; ++t) {
                double v = (t <= i + j ? pa * E[i][j][t] : 0.0) + (t + 1 <= i + j ? (t + 1) * E[i][j][t + 1] : 0.0);
                if (t > 0) v += h * E[i][j][t - 1];
                E[i + 1][j][t] = v;
            }
}

// sum_{t<=tx,u<=ty,v<=tz} ex[t] ey[u] ez[v] R_tuv, R scaled by sc (-2a)^n F_n(T)
__device__ double herm_contract(const double *ex, const double *ey, const double *ez, int tx, int ty, int tz,
                                double sc, double a, double X, double Y, double Z)
{
    const int L = tx + ty + tz;
    double F[16];
    boys(L, a * (X * X + Y * Y + Z * Z), F);
    const int dy = tz + 1, dx = (ty + 1) * dy;
    double bufA[64], bufB[64];
    double *cur = bufA, *nxt = bufB;
    // level n = L: only R_000
    for (int n = L; n >= 0; --n) {
        double base = sc * F[n];
        for (int k = 0; k < n; ++k) base *= -2.0 * a;
        const int top = L - n;
        for (int t = 0; t <= tx; ++t)
            for (int u = 0; u <= ty; ++u)
                for (int v = 0; v <= tz; ++v) {
                    const int idx = t * dx + u * dy + v;
                    if (t + u + v > top) continue;
                    double r;
                    if (t + u + v == 0) {
                        r = base;
                    } else if (t > 0) {
                        r = X * nxt[(t - 1) * dx + u * dy + v];
                        if (t > 1) r += (t - 1) * nxt[(t - 2) * dx + u * dy + v];
                    } else if (u > 0) {
                        r = Y * nxt[u * dy - dy + v];
                        if (u > 1) r += (u - 1) * nxt[(u - 2) * dy + v];
                    } else {
                        r = Z * nxt[v - 1];
                        if (v > 1) r += (v - 1) * nxt[v - 2];
                    }
                    cur[idx] = r;
                }
        double *tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    // after the loop the level-0 values are in nxt
    double s = 0.0;
    for (int t = 0; t <= tx; ++t)
        for (int u = 0; u <= ty; ++u)
            for (int v = 0; v <= tz; ++v) s += ex[t] * ey[u] * ez[v] * nxt[t * dx + u * dy + v];
    return s;
}

__global__ void onebody_kernel(const OneArgs a)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= a.nitem) return;
    const int ish = a.item[5 * it], jsh = a.item[5 * it + 1], ia = a.item[5 * it + 2], ib = a.item[5 * it + 3];
    const int ij = a.item[5 * it + 4];
    const int la = a.l[ish], lb = a.l[jsh];
    const int ca = c_cart1[la][ia], cb = c_cart1[lb][ib];
    const int ex[3] = {ca & 15, (ca >> 4) & 15, ca >> 8};
    const int eb[3] = {cb & 15, (cb >> 4) & 15, cb >> 8};
    const double *A = a.xyz + 3 * a.cen[ish], *B = a.xyz + 3 * a.cen[jsh];
    const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double nrm = c_norm1[la][ia] * c_norm1[lb][ib];
    const double SR = 34.98683665524972497;        // 2 pi^(5/2)
    const double PI32 = 5.568327996831707845;      // pi^(3/2)
    double sv = 0.0, tv = 0.0, vv = 0.0, dv = 0.0;
    double E[3][EM][EM][ET];
    for (int i = a.poff[ish]; i < a.poff[ish + 1]; ++i)
        for (int j = a.poff[jsh]; j < a.poff[jsh + 1]; ++j) {
            const double ea = a.al[i], ebx = a.al[j], p = ea + ebx, c12 = a.co[i] * a.co[j];
            const double kab = exp(-ea * ebx * ab2 / p);
            double P[3];
            for (int d = 0; d < 3; ++d) {
                P[d] = (ea * A[d] + ebx * B[d]) / p;
                herm_e(E[d], ex[d] + 1, eb[d] + 1, 0.5 / p, P[d] - A[d], P[d] - B[d]);
            }
            if (a.S) {
                const double s12 = PI32 * kab / (p * sqrt(p));
                const double e0 = E[0][ex[0]][eb[0]][0] * E[1][ex[1]][eb[1]][0] * E[2][ex[2]][eb[2]][0];
                sv += c12 * nrm * s12 * e0;
                double kin = 0.0;
                for (int d = 0; d < 3; ++d) {
                    const int i1 = ex[d], j1 = eb[d];
                    double td = 2.0 * ea * ebx * E[d][i1 + 1][j1 + 1][0];
                    if (i1) td -= i1 * ebx * E[d][i1 - 1][j1 + 1][0];
                    if (j1) {
                        td -= j1 * ea * E[d][i1 + 1][j1 - 1][0];
                        if (i1) td += 0.5 * i1 * j1 * E[d][i1 - 1][j1 - 1][0];
                    }
                    double o = 1.0;
                    for (int d2 = 0; d2 < 3; ++d2)
                        if (d2 != d) o *= E[d2][ex[d2]][eb[d2]][0];
                    kin += td * o;
                }
                tv += c12 * nrm * s12 * kin;
                const double sr = 2.0 * s12 * sqrt(p / 3.14159265358979323846);
                for (int c = 0; c < a.ncen; ++c) {
                    if (c == a.skipcen || a.q[c] == 0.0) continue;
                    const double *C = a.xyz + 3 * c;
                    vv -= c12 * nrm * a.q[c] *
                          herm_contract(E[0][ex[0]][eb[0]], E[1][ex[1]][eb[1]], E[2][ex[2]][eb[2]], ex[0] + eb[0],
                                        ex[1] + eb[1], ex[2] + eb[2], sr, p, P[0] - C[0], P[1] - C[1], P[2] - C[2]);
                }
            }
            if (a.V) {
                const double *Q = a.xyz + 3 * a.skipcen;
                for (int g = 0; g < 6; ++g) {
                    const double qx = c_palf[g], tx = p + qx;
                    const double sr = 2.0 * c12 * c_pcof[g] * SR * kab * (0.5 / p) * (1.0 / qx) / sqrt(tx);
                    const double w = p * qx / tx;
                    dv += nrm * herm_contract(E[0][ex[0]][eb[0]], E[1][ex[1]][eb[1]], E[2][ex[2]][eb[2]],
                                              ex[0] + eb[0], ex[1] + eb[1], ex[2] + eb[2], sr, w, P[0] - Q[0],
                                              P[1] - Q[1], P[2] - Q[2]);
                }
            }
        }
    if (a.S) {
        a.S[ij] = sv;
        a.T[ij] = tv;
        a.H[ij] = tv + vv;
    }
    if (a.V) a.V[ij] = dv;
}

// ------------------------------------------------------------- moments
// Dipole and quadrupole integrals about the coordinate origin (the
// quantities momints.c:13-85 forms), one thread per component pair.  With
// the Hermite expansion of the pair about P, the one-dimensional moments are
//   M0 = E_0,  M1 = E_1 + P E_0,  M2 = 2 E_2 + 2 P E_1 + (P^2 + 1/(2p)) E_0
// (times sqrt(pi/p)), and a three-dimensional moment is the product of the
// per-direction factors: x = M1x M0y M0z, xy = M1x M1y M0z, xx = M2x M0y M0z.
struct MomArgs {
    const int *item;     // per thread: ish, jsh, ia, ib, packed index
    int nitem;
    const int *l, *cen, *poff;
    const double *al, *co, *xyz;
    size_t no2;
    double *out;         // [9][no2]: x, y, z, then xx, xy, xz, yy, yz, zz
};

__global__ void moments_kernel(const MomArgs a)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= a.nitem) return;
    const int ish = a.item[5 * it], jsh = a.item[5 * it + 1], ia = a.item[5 * it + 2], ib = a.item[5 * it + 3];
    const int ij = a.item[5 * it + 4];
    const int la = a.l[ish], lb = a.l[jsh];
    const int ca = c_cart1[la][ia], cb = c_cart1[lb][ib];
    const int ex[3] = {ca & 15, (ca >> 4) & 15, ca >> 8};
    const int eb[3] = {cb & 15, (cb >> 4) & 15, cb >> 8};
    const double *A = a.xyz + 3 * a.cen[ish], *B = a.xyz + 3 * a.cen[jsh];
    const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double nrm = c_norm1[la][ia] * c_norm1[lb][ib];
    const double PI32 = 5.568327996831707845;      // pi^(3/2)
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double E[3][EM][EM][ET];
    for (int i = a.poff[ish]; i < a.poff[ish + 1]; ++i)
        for (int j = a.poff[jsh]; j < a.poff[jsh + 1]; ++j) {
            const double ea = a.al[i], ebx = a.al[j], p = ea + ebx;
            const double w = a.co[i] * a.co[j] * nrm * PI32 * exp(-ea * ebx * ab2 / p) / (p * sqrt(p));
            double m0[3], m1[3], m2[3];
            for (int d = 0; d < 3; ++d) {
                const double P = (ea * A[d] + ebx * B[d]) / p;
                // E up to t = ex + eb + 2, zero above ex + eb
                herm_e(E[d], ex[d] + 1, eb[d] + 1, 0.5 / p, P - A[d], P - B[d]);
                const double *e = E[d][ex[d]][eb[d]];
                m0[d] = e[0];
                m1[d] = e[1] + P * e[0];
                m2[d] = 2.0 * e[2] + 2.0 * P * e[1] + (P * P + 0.5 / p) * e[0];
            }
            acc[0] += w * m1[0] * m0[1] * m0[2];
            acc[1] += w * m0[0] * m1[1] * m0[2];
            acc[2] += w * m0[0] * m0[1] * m1[2];
            acc[3] += w * m2[0] * m0[1] * m0[2];
            acc[4] += w * m1[0] * m1[1] * m0[2];
            acc[5] += w * m1[0] * m0[1] * m1[2];
            acc[6] += w * m0[0] * m2[1] * m0[2];
            acc[7] += w * m0[0] * m1[1] * m1[2];
            acc[8] += w * m0[0] * m0[1] * m2[2];
        }
    for (int k = 0; k < 9; ++k) a.out[k * a.no2 + ij] = acc[k];
}

int run_moments(int nsh, const int *l, const int *cen, const int *off, const int *nst, const int *poff,
                const double *al, const double *co, int ncen, const double *xyz, int n, double *dip, double *quad,
                cudaStream_t s)
{
    std::vector<int> items;
    for (int i = 0; i < nsh; ++i) {
        if (!nst[i]) continue;
        for (int j = 0; j <= i; ++j) {
            if (!nst[j]) continue;
            for (int ia = 0; ia < nst[i]; ++ia)
                for (int ib = 0; ib < nst[j]; ++ib) {
                    const int ir = off[i] + ia, jr = off[j] + ib;
                    if (jr > ir) continue;
                    items.insert(items.end(), {i, j, ia, ib, ir * (ir + 1) / 2 + jr});
                }
        }
    }
    const int nitem = (int)items.size() / 5;
    const size_t no2 = (size_t)n * (n + 1) / 2;
    const int np = poff[nsh];
    void *d_item = nullptr, *d_l = nullptr, *d_cen = nullptr, *d_poff = nullptr, *d_al = nullptr, *d_co = nullptr,
         *d_xyz = nullptr, *d_out = nullptr;
    cudaError_t e = cudaSuccess;
    auto up = [&](void **d, const void *h, size_t b) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(d, b ? b : 16);
        if (e == cudaSuccess && b) e = cudaMemcpyAsync(*d, h, b, cudaMemcpyHostToDevice, s);
    };
    up(&d_item, items.data(), sizeof(int) * items.size());
    up(&d_l, l, sizeof(int) * nsh);
    up(&d_cen, cen, sizeof(int) * nsh);
    up(&d_poff, poff, sizeof(int) * (nsh + 1));
    up(&d_al, al, sizeof(double) * np);
    up(&d_co, co, sizeof(double) * np);
    up(&d_xyz, xyz, sizeof(double) * 3 * ncen);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(double) * no2 * 9);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, sizeof(double) * no2 * 9, s);
    if (e == cudaSuccess && nitem) {
        MomArgs a{};
        a.item = (const int *)d_item;
        a.nitem = nitem;
        a.l = (const int *)d_l;
        a.cen = (const int *)d_cen;
        a.poff = (const int *)d_poff;
        a.al = (const double *)d_al;
        a.co = (const double *)d_co;
        a.xyz = (const double *)d_xyz;
        a.no2 = no2;
        a.out = (double *)d_out;
        moments_kernel<<<(nitem + 127) / 128, 128, 0, s>>>(a);
        e = cudaGetLastError();
    }
    std::vector<double> h(no2 * 9);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_out, sizeof(double) * no2 * 9, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (void *p : {d_item, d_l, d_cen, d_poff, d_al, d_co, d_xyz, d_out})
        if (p) cudaFree(p);
    if (e != cudaSuccess) return fail(PATGPU_ECUDA, "moment integrals: %s", cudaGetErrorString(e));
    for (size_t k = 0; k < 3 * no2; ++k) dip[k] = h[k];
    for (size_t k = 0; k < 6 * no2; ++k) quad[k] = h[3 * no2 + k];
    return 0;
}

int run_oneints(int nsh, const int *l, const int *cen, const int *off, const int *nst, const int *poff,
                const double *al, const double *co, int ncen, const double *q, const double *xyz, int skipcen,
                int n, double *S, double *T, double *H, double *Hdpm, cudaStream_t s)
{
    std::vector<int> items;
    for (int i = 0; i < nsh; ++i) {
        if (!nst[i]) continue;
        for (int j = 0; j <= i; ++j) {
            if (!nst[j]) continue;
            for (int ia = 0; ia < nst[i]; ++ia)
                for (int ib = 0; ib < nst[j]; ++ib) {
                    const int ir = off[i] + ia, jr = off[j] + ib;
                    if (jr > ir) continue;
                    items.insert(items.end(), {i, j, ia, ib, ir * (ir + 1) / 2 + jr});
                }
        }
    }
    if (Hdpm && (skipcen < 0 || skipcen >= ncen))
        return fail(PATGPU_EINVAL, "DPM needs the positron centre (skipcen=%d, ncen=%d)", skipcen, ncen);
    const int nitem = (int)items.size() / 5;
    const size_t no2 = (size_t)n * (n + 1) / 2;
    const int np = poff[nsh];
    void *d_item = nullptr, *d_l = nullptr, *d_cen = nullptr, *d_poff = nullptr, *d_al = nullptr, *d_co = nullptr,
         *d_q = nullptr, *d_xyz = nullptr, *d_out = nullptr;
    cudaError_t e = cudaSuccess;
    auto up = [&](void **d, const void *h, size_t b) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(d, b ? b : 16);
        if (e == cudaSuccess && b) e = cudaMemcpyAsync(*d, h, b, cudaMemcpyHostToDevice, s);
    };
    up(&d_item, items.data(), sizeof(int) * items.size());
    up(&d_l, l, sizeof(int) * nsh);
    up(&d_cen, cen, sizeof(int) * nsh);
    up(&d_poff, poff, sizeof(int) * (nsh + 1));
    up(&d_al, al, sizeof(double) * np);
    up(&d_co, co, sizeof(double) * np);
    up(&d_q, q, sizeof(double) * ncen);
    up(&d_xyz, xyz, sizeof(double) * 3 * ncen);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(double) * no2 * 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, sizeof(double) * no2 * 4, s);
    if (e == cudaSuccess && nitem) {
        OneArgs a{};
        a.item = (const int *)d_item;
        a.nitem = nitem;
        a.l = (const int *)d_l;
        a.cen = (const int *)d_cen;
        a.poff = (const int *)d_poff;
        a.al = (const double *)d_al;
        a.co = (const double *)d_co;
        a.q = (const double *)d_q;
        a.xyz = (const double *)d_xyz;
        a.ncen = ncen;
        a.skipcen = skipcen;
        double *o = (double *)d_out;
        if (S) {
            a.S = o;
            a.T = o + no2;
            a.H = o + 2 * no2;
        }
        if (Hdpm) a.V = o + 3 * no2;
        onebody_kernel<<<(nitem + 127) / 128, 128, 0, s>>>(a);
        e = cudaGetLastError();
    }
    std::vector<double> h(no2 * 4);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_out, sizeof(double) * no2 * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (void *p : {d_item, d_l, d_cen, d_poff, d_al, d_co, d_q, d_xyz, d_out})
        if (p) cudaFree(p);
    if (e != cudaSuccess) return fail(PATGPU_ECUDA, "one-body integrals: %s", cudaGetErrorString(e));
    if (S)
        for (size_t k = 0; k < no2; ++k) {
            S[k] = h[k];
            T[k] = h[no2 + k];
            H[k] = h[2 * no2 + k];
        }
    if (Hdpm)
        for (size_t k = 0; k < no2; ++k) Hdpm[k] -= h[3 * no2 + k];
    return 0;
}

// ------------------------------------------------------------ gradient
// Nuclear-coordinate derivatives of the one-body terms of the closed-shell
// energy E = 2 tr(P H) + ... - 2 tr(W S) contributions, with the half
// density P and the energy-weighted density W = sum_occ e_i c_i c_i^T
// (packed).  Per primitive of exponent alpha a basis function moves with its
// centre as d phi_a / dA_x = 2 alpha phi_{a+1x} - a_x phi_{a-1x}; S and T
// depend on A - B only (dB = -dA); the attraction to a charge at C gives
// dC from the Hermite integrals directly, d R_tuv / dC_x = -R_{t+1,u,v},
// and dB = -(dA + dC).  The DPM Gaussians of dpmints.c:30-36 sit at the
// positron centre and enter H with a minus sign (dpmints.c:187).

struct OneGradArgs {
    const int *item;
    int nitem;
    const int *l, *cen, *poff, *off;
    const double *al, *co, *q, *xyz;
    int ncen, skipcen, with_dpm;
    const double *P, *W;   // packed half density and energy-weighted density
    double *grad;          // [ncen][3]
};

// Level-0 Hermite Coulomb integrals sc * R_tuv(a; X, Y, Z) for t <= tx,
// u <= ty, v <= tz, stored at R[(t (ty+1) + u)(tz+1) + v]; the cube has at
// most 64 entries.
__device__ void herm_r(int tx, int ty, int tz, double sc, double a, double X, double Y, double Z, double *R)
{
    const int L = tx + ty + tz;
    double F[16];
    boys(L, a * (X * X + Y * Y + Z * Z), F);
    const int dy = tz + 1, dx = (ty + 1) * dy;
    double bufA[64], bufB[64];
    double *cur = bufA, *nxt = bufB;
    for (int n = L; n >= 0; --n) {
        double base = sc * F[n];
        for (int k = 0; k < n; ++k) base *= -2.0 * a;
        const int top = L - n;
        for (int t = 0; t <= tx; ++t)
            for (int u = 0; u <= ty; ++u)
                for (int v = 0; v <= tz; ++v) {
                    if (t + u + v > top) continue;
                    double r;
                    if (t + u + v == 0) {
                        r = base;
                    } else if (t > 0) {
                        r = X * nxt[(t - 1) * dx + u * dy + v];
                        if (t > 1) r += (t - 1) * nxt[(t - 2) * dx + u * dy + v];
                    } else if (u > 0) {
                        r = Y * nxt[(u - 1) * dy + v];
                        if (u > 1) r += (u - 1) * nxt[(u - 2) * dy + v];
                    } else {
                        r = Z * nxt[v - 1];
                        if (v > 1) r += (v - 1) * nxt[v - 2];
                    }
                    cur[t * dx + u * dy + v] = r;
                }
        double *tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    for (int k = 0; k < (tx + 1) * dx; ++k) R[k] = nxt[k];
}

// sum_{t,u,v} ex[t] ey[u] ez[v] R[t+sx][u+sy][v+sz]
__device__ __forceinline__ double herm_dot(const double *ex, const double *ey, const double *ez, int nx, int ny,
                                           int nz, const double *R, int dx, int dy, int sx, int sy, int sz)
{
    double s = 0.0;
    for (int t = 0; t <= nx; ++t)
        for (int u = 0; u <= ny; ++u) {
            double su = 0.0;
            for (int v = 0; v <= nz; ++v) su += ez[v] * R[(t + sx) * dx + (u + sy) * dy + v + sz];
            s += ex[t] * ey[u] * su;
        }
    return s;
}

#define EG 6
// kinetic factor of one direction (the product rule of oneints.c:81-116)
__device__ __forceinline__ double kin_dir(double E[EG][EG][ET], int i, int j, double a, double b)
{
    double td = 2.0 * a * b * E[i + 1][j + 1][0];
    if (i) td -= i * b * E[i - 1][j + 1][0];
    if (j) {
        td -= j * a * E[i + 1][j - 1][0];
        if (i) td += 0.5 * i * j * E[i - 1][j - 1][0];
    }
    return td;
}

__device__ double kin3(double E[3][EG][EG][ET], const int *i3, const int *j3, double a, double b)
{
    double k = 0.0;
    for (int d = 0; d < 3; ++d) {
        double o = kin_dir(E[d], i3[d], j3[d], a, b);
        for (int d2 = 0; d2 < 3; ++d2)
            if (d2 != d) o *= E[d2][i3[d2]][j3[d2]][0];
        k += o;
    }
    return k;
}

// Derivatives of the attraction to one Gaussian-smeared or point charge at
// C (scaled by pre; R with exponent w): dA (raised/lowered bra) and dC.
__device__ void attraction_deriv(double E[3][EG][EG][ET], const int *ea, const int *eb, double alpha,
                                 double pre, double w, const double *P, const double *C, double *dA, double *dC)
{
    const int tx = ea[0] + eb[0] + 1, ty = ea[1] + eb[1] + 1, tz = ea[2] + eb[2] + 1;
    double R[64];
    herm_r(tx, ty, tz, pre, w, P[0] - C[0], P[1] - C[1], P[2] - C[2], R);
    const int dy = tz + 1, dx = (ty + 1) * dy;
    const double *e0[3] = {E[0][ea[0]][eb[0]], E[1][ea[1]][eb[1]], E[2][ea[2]][eb[2]]};
    for (int d = 0; d < 3; ++d) {
        const int n0 = ea[0] + eb[0], n1 = ea[1] + eb[1], n2 = ea[2] + eb[2];
        // dC: R shifted by one in direction d
        dC[d] = -herm_dot(e0[0], e0[1], e0[2], n0, n1, n2, R, dx, dy, d == 0, d == 1, d == 2);
        // dA: raised and lowered bra exponent in direction d
        const double *ep[3] = {e0[0], e0[1], e0[2]};
        int np[3] = {n0, n1, n2};
        ep[d] = E[d][ea[d] + 1][eb[d]];
        np[d] += 1;
        double v = 2.0 * alpha * herm_dot(ep[0], ep[1], ep[2], np[0], np[1], np[2], R, dx, dy, 0, 0, 0);
        if (ea[d] > 0) {
            ep[d] = E[d][ea[d] - 1][eb[d]];
            np[d] -= 2;
            v -= ea[d] * herm_dot(ep[0], ep[1], ep[2], np[0], np[1], np[2], R, dx, dy, 0, 0, 0);
        }
        dA[d] = v;
    }
}

__global__ void onebody_grad_kernel(const OneGradArgs a)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= a.nitem) return;
    const int ish = a.item[5 * it], jsh = a.item[5 * it + 1], ia = a.item[5 * it + 2], ib = a.item[5 * it + 3];
    const int ij = a.item[5 * it + 4];
    const int ir = a.off[ish] + ia, jr = a.off[jsh] + ib;
    const double fac = ir == jr ? 1.0 : 2.0;
    const double wP = 2.0 * fac * a.P[ij];
    const double wW = a.W ? -2.0 * fac * a.W[ij] : 0.0;
    const int la = a.l[ish], lb = a.l[jsh];
    const int ca = c_cart1[la][ia], cb = c_cart1[lb][ib];
    const int ex[3] = {ca & 15, (ca >> 4) & 15, ca >> 8};
    const int eb[3] = {cb & 15, (cb >> 4) & 15, cb >> 8};
    const int cenA = a.cen[ish], cenB = a.cen[jsh];
    const double *A = a.xyz + 3 * cenA, *B = a.xyz + 3 * cenB;
    const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double nrm = c_norm1[la][ia] * c_norm1[lb][ib];
    const double SR = 34.98683665524972497;        // 2 pi^(5/2)
    const double PI32 = 5.568327996831707845;      // pi^(3/2)
    double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
    double E[3][EG][EG][ET];
    for (int i = a.poff[ish]; i < a.poff[ish + 1]; ++i)
        for (int j = a.poff[jsh]; j < a.poff[jsh + 1]; ++j) {
            const double ea = a.al[i], ebx = a.al[j], p = ea + ebx, c12 = a.co[i] * a.co[j];
            const double kab = exp(-ea * ebx * ab2 / p);
            double P[3];
            for (int d = 0; d < 3; ++d) {
                P[d] = (ea * A[d] + ebx * B[d]) / p;
                herm_e<EG>(E[d], ex[d] + 2, eb[d] + 1, 0.5 / p, P[d] - A[d], P[d] - B[d]);
            }
            const double s12 = PI32 * kab / (p * sqrt(p));
            const double pre = c12 * nrm * s12;
            // overlap and kinetic: dB = -dA
            for (int d = 0; d < 3; ++d) {
                double o = 1.0;
                for (int d2 = 0; d2 < 3; ++d2)
                    if (d2 != d) o *= E[d2][ex[d2]][eb[d2]][0];
                double dS = 2.0 * ea * E[d][ex[d] + 1][eb[d]][0];
                if (ex[d]) dS -= ex[d] * E[d][ex[d] - 1][eb[d]][0];
                dS *= o;
                int up[3] = {ex[0], ex[1], ex[2]};
                up[d] += 1;
                double dT = 2.0 * ea * kin3(E, up, eb, ea, ebx);
                if (ex[d]) {
                    up[d] -= 2;
                    dT -= ex[d] * kin3(E, up, eb, ea, ebx);
                }
                const double g = pre * (wW * dS + wP * dT);
                gA[d] += g;
                gB[d] -= g;
            }
            // nuclear attraction (every charged centre but the positron)
            const double sr = 2.0 * s12 * sqrt(p / 3.14159265358979323846);
            for (int c = 0; c < a.ncen; ++c) {
                if (c == a.skipcen || a.q[c] == 0.0) continue;
                double dA[3], dC[3];
                attraction_deriv(E, ex, eb, ea, -c12 * nrm * a.q[c] * sr, p, P, a.xyz + 3 * c, dA, dC);
                for (int d = 0; d < 3; ++d) {
                    gA[d] += wP * dA[d];
                    gB[d] -= wP * (dA[d] + dC[d]);
                    atomicAdd(a.grad + 3 * c + d, wP * dC[d]);
                }
            }
            // DPM potential at the positron centre, H -= V_DPM
            if (a.with_dpm) {
                const double *Q = a.xyz + 3 * a.skipcen;
                double gQ[3] = {0, 0, 0};
                for (int g = 0; g < 6; ++g) {
                    const double qx = c_palf[g], tx = p + qx;
                    const double sg = 2.0 * c12 * c_pcof[g] * SR * kab * (0.5 / p) * (1.0 / qx) / sqrt(tx);
                    double dA[3], dC[3];
                    attraction_deriv(E, ex, eb, ea, -nrm * sg, p * qx / tx, P, Q, dA, dC);
                    for (int d = 0; d < 3; ++d) {
                        gA[d] += wP * dA[d];
                        gB[d] -= wP * (dA[d] + dC[d]);
                        gQ[d] += wP * dC[d];
                    }
                }
                for (int d = 0; d < 3; ++d) atomicAdd(a.grad + 3 * a.skipcen + d, gQ[d]);
            }
        }
    for (int d = 0; d < 3; ++d) {
        atomicAdd(a.grad + 3 * cenA + d, gA[d]);
        atomicAdd(a.grad + 3 * cenB + d, gB[d]);
    }
}

int run_onebody_grad(int nsh, const int *l, const int *cen, const int *off, const int *nst, const int *poff,
                     const double *al, const double *co, int ncen, const double *q, const double *xyz, int skipcen,
                     int n, const double *P, const double *W, int with_dpm, double *grad, cudaStream_t s)
{
    if (with_dpm && (skipcen < 0 || skipcen >= ncen))
        return fail(PATGPU_EINVAL, "DPM needs the positron centre (skipcen=%d, ncen=%d)", skipcen, ncen);
    std::vector<int> items;
    for (int i = 0; i < nsh; ++i) {
        if (!nst[i]) continue;
        for (int j = 0; j <= i; ++j) {
            if (!nst[j]) continue;
            for (int ia = 0; ia < nst[i]; ++ia)
                for (int ib = 0; ib < nst[j]; ++ib) {
                    const int ir = off[i] + ia, jr = off[j] + ib;
                    if (jr > ir) continue;
                    items.insert(items.end(), {i, j, ia, ib, ir * (ir + 1) / 2 + jr});
                }
        }
    }
    const int nitem = (int)items.size() / 5;
    const size_t no2 = (size_t)n * (n + 1) / 2;
    const int np = poff[nsh];
    void *d_item = nullptr, *d_l = nullptr, *d_cen = nullptr, *d_poff = nullptr, *d_off = nullptr, *d_al = nullptr,
         *d_co = nullptr, *d_q = nullptr, *d_xyz = nullptr, *d_P = nullptr, *d_W = nullptr, *d_g = nullptr;
    cudaError_t e = cudaSuccess;
    auto up = [&](void **d, const void *h, size_t b) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(d, b ? b : 16);
        if (e == cudaSuccess && b) e = cudaMemcpyAsync(*d, h, b, cudaMemcpyHostToDevice, s);
    };
    up(&d_item, items.data(), sizeof(int) * items.size());
    up(&d_l, l, sizeof(int) * nsh);
    up(&d_cen, cen, sizeof(int) * nsh);
    up(&d_poff, poff, sizeof(int) * (nsh + 1));
    up(&d_off, off, sizeof(int) * nsh);
    up(&d_al, al, sizeof(double) * np);
    up(&d_co, co, sizeof(double) * np);
    up(&d_q, q, sizeof(double) * ncen);
    up(&d_xyz, xyz, sizeof(double) * 3 * ncen);
    up(&d_P, P, sizeof(double) * no2);
    if (W) up(&d_W, W, sizeof(double) * no2);
    if (e == cudaSuccess) e = cudaMalloc(&d_g, sizeof(double) * 3 * ncen);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_g, 0, sizeof(double) * 3 * ncen, s);
    if (e == cudaSuccess && nitem) {
        OneGradArgs a{};
        a.item = (const int *)d_item;
        a.nitem = nitem;
        a.l = (const int *)d_l;
        a.cen = (const int *)d_cen;
        a.poff = (const int *)d_poff;
        a.off = (const int *)d_off;
        a.al = (const double *)d_al;
        a.co = (const double *)d_co;
        a.q = (const double *)d_q;
        a.xyz = (const double *)d_xyz;
        a.ncen = ncen;
        a.skipcen = skipcen;
        a.with_dpm = with_dpm;
        a.P = (const double *)d_P;
        a.W = (const double *)d_W;
        a.grad = (double *)d_g;
        onebody_grad_kernel<<<(nitem + 63) / 64, 64, 0, s>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, d_g, sizeof(double) * 3 * ncen, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (void *p : {d_item, d_l, d_cen, d_poff, d_off, d_al, d_co, d_q, d_xyz, d_P, d_W, d_g})
        if (p) cudaFree(p);
    if (e != cudaSuccess) return fail(PATGPU_ECUDA, "one-body gradient: %s", cudaGetErrorString(e));
    return 0;
}

}  // namespace pg
