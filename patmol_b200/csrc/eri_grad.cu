// eri_grad.cu -- the derivative-ERI gradient kernel (see eri_grad.cuh for
// the mathematics).
//
// GPU mapping: a team of TQ lanes owns one shell quartet, as in the
// shared-memory Fock kernel.  Per quartet the team forms the weights
// deg * Gamma * (component factors of basis.c:309-319) in shared memory;
// per primitive quartet it evaluates the Rys rule, lanes j < 3n build the
// 2-D recursion (rys.c:2269-2293) for one root and direction in shared
// memory, all lanes then transfer it (rys.c:2295-2336) to the extended 1-D
// table I[a][b][c][d] with a <= la+1, b <= lb+1, c <= lc+1, d <= ld, one
// table entry per lane at a time; then every lane walks its
// Cartesian components and accumulates nine sums (centres A, B, C times
// x, y, z).  The team reduces them and adds twelve numbers into the
// gradient with FP64 atomics.  The class is a runtime argument: the
// gradient is evaluated once per geometry, so one kernel serves all 55
// classes instead of 55 instantiations.
#include "eri_grad.cuh"

namespace pg {

extern __constant__ RysConst c_rys;
extern __constant__ int c_cart[4][10];
extern __constant__ double c_norm[4][10];

namespace {

constexpr double kSRg = 34.98683665524972497;   // 2 pi^(5/2)
constexpr int kRysDegG = 11;                    // degree of the Chebyshev pieces (rys_table.h)
constexpr int kBlk = 128;

struct GradDims {
    int la, lb, lc, ld, na, nb, nc, nd, ncart;
    int nr, l12, l34, ea, eb, ec, ed, tsz, gsz;
    int tq, nteam, rw, team;   // team: doubles of shared memory per team
};

// Lanes per team: the transfer and contraction phases spread over all of
// them, so mid-size classes take whole warps and large ones a block.
int tq_for(int ncart)
{
    return ncart <= 300 ? 32 : ncart <= 1500 ? 64 : 128;
}

GradDims grad_dims(int la, int lb, int lc, int ld)
{
    GradDims d{};
    d.la = la; d.lb = lb; d.lc = lc; d.ld = ld;
    d.na = (la + 1) * (la + 2) / 2;
    d.nb = (lb + 1) * (lb + 2) / 2;
    d.nc = (lc + 1) * (lc + 2) / 2;
    d.nd = (ld + 1) * (ld + 2) / 2;
    d.ncart = d.na * d.nb * d.nc * d.nd;
    d.nr = (la + lb + lc + ld + 1) / 2 + 1;
    d.l12 = la + lb + 1;
    d.l34 = lc + ld + 1;
    d.ea = la + 2; d.eb = lb + 2; d.ec = lc + 2; d.ed = ld + 1;
    d.tsz = d.ea * d.eb * d.ec * d.ed;
    d.gsz = (d.l12 + 1) * (d.l34 + 1);
    d.tq = tq_for(d.ncart);
    d.nteam = kBlk / d.tq;
    d.rw = (2 * d.nr + 1) / 2 * 2;
    d.team = (d.rw + 3 * d.nr * d.gsz + 3 * d.nr * d.tsz + d.ncart + 9 * d.tq + 1) / 2 * 2;
    return d;
}

// 2-D recursion into G[i * W + j] (W = l34 + 1) for i <= l12, j <= l34.
__device__ __forceinline__ void grad_vrr(double *G, int l12, int l34, double g00, double B00, double B10,
                                         double B01, double C, double Cp)
{
    const int W = l34 + 1;
    G[0] = g00;
    G[W] = C * g00;
    for (int i = 1; i < l12; ++i) G[(i + 1) * W] = i * B10 * G[(i - 1) * W] + C * G[i * W];
    for (int j = 0; j < l34; ++j)
        for (int i = 0; i <= l12; ++i) {
            double v = Cp * G[i * W + j];
            if (j > 0) v = fma(j * B01, G[i * W + j - 1], v);
            if (i > 0) v = fma(i * B00, G[(i - 1) * W + j], v);
            G[i * W + j + 1] = v;
        }
}

__global__ void __launch_bounds__(kBlk, 4) eri_grad_kernel(const EriArgs args, const GradArgs ga, const GradDims dm)
{
    extern __shared__ double smem[];
    __shared__ int s_np[kBlk / 8];
    __shared__ int s_maxp;

    const int TQ = dm.tq, NTEAM = dm.nteam, NR = dm.nr, TSZ = dm.tsz;
    const int NB = dm.nb, NC = dm.nc, ND = dm.nd, NCART = dm.ncart;
    const int SA = dm.eb * dm.ec * dm.ed, SB = dm.ec * dm.ed, SC = dm.ed;   // table strides of a, b, c
    const int team = threadIdx.x / TQ, lane = threadIdx.x % TQ;
    double *s_rw = smem + (size_t)team * dm.team;   // nodes [0, NR), weights [NR, 2NR)
    double *s_G = s_rw + dm.rw;                     // [3][NR][gsz] 2-D recursion
    double *s_tab = s_G + 3 * NR * dm.gsz;          // [3][TSZ][NR]
    double *s_gam = s_tab + 3 * NR * TSZ;           // [NCART]
    double *s_red = s_gam + NCART;                  // [9][TQ]
    const int n = args.n;
    const double *__restrict__ P = args.D0;

    for (long long base = (long long)blockIdx.x * NTEAM; base < args.nquart;
         base += (long long)gridDim.x * NTEAM) {
        const long long qi = base + team;
        int u = 0, v = 0, npb = 0, npk = 0, pb0 = 0, pk0 = 0;
        const bool active = qi < args.nquart && eri_quartet_at(args, qi, u, v);
        double ax = 0, ay = 0, az = 0, abx = 0, aby = 0, abz = 0;
        double cx = 0, cy = 0, cz = 0, cdx = 0, cdy = 0, cdz = 0;
        if (active) {
            npb = args.pr.pnum[u];
            npk = args.pr.pnum[v];
            pb0 = args.pr.pstart[u];
            pk0 = args.pr.pstart[v];
            ax = args.pr.ax[u]; ay = args.pr.ay[u]; az = args.pr.az[u];
            abx = args.pr.abx[u]; aby = args.pr.aby[u]; abz = args.pr.abz[u];
            cx = args.pr.ax[v]; cy = args.pr.ay[v]; cz = args.pr.az[v];
            cdx = args.pr.abx[v]; cdy = args.pr.aby[v]; cdz = args.pr.abz[v];
            const int fa = args.pr.fa[u], fb = args.pr.fb[u], fc = args.pr.fa[v], fd = args.pr.fb[v];
            const bool sab = args.pr.sa[u] == args.pr.sb[u], scd = args.pr.sa[v] == args.pr.sb[v];
            const double deg = (sab ? 1.0 : 2.0) * (scd ? 1.0 : 2.0) * (u == v ? 1.0 : 2.0);
            for (int c = lane; c < NCART; c += TQ) {
                const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
                const int i = fa + ia, j = fb + ib, k = fc + ic, l = fd + id;
                const double g = 2.0 * __ldg(P + (size_t)i * n + j) * __ldg(P + (size_t)k * n + l) -
                                 0.5 * (__ldg(P + (size_t)i * n + k) * __ldg(P + (size_t)j * n + l) +
                                        __ldg(P + (size_t)i * n + l) * __ldg(P + (size_t)j * n + k));
                s_gam[c] = deg * g * c_norm[dm.la][ia] * c_norm[dm.lb][ib] * c_norm[dm.lc][ic] * c_norm[dm.ld][id];
            }
        }
        if (lane == 0) s_np[team] = active ? npb * npk : 0;
        __syncthreads();
        if (threadIdx.x == 0) {
            int m = 0;
            for (int t = 0; t < NTEAM; ++t) m = max(m, s_np[t]);
            s_maxp = m;
        }
        __syncthreads();
        const int maxp = s_maxp;
        double g[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) g[k] = 0.0;

        for (int ip = 0; ip < maxp; ++ip) {
            bool work = active && ip < npb * npk;
            double p = 1, q = 1, sr = 0, pax = 0, pay = 0, paz = 0, qcx = 0, qcy = 0, qcz = 0;
            double pqx = 0, pqy = 0, pqz = 0, alpha = 0, beta = 0, gamma = 0;
            if (work) {
                const int ib = pb0 + ip / npk, ik = pk0 + ip % npk;
                p = args.pp.p[ib];
                q = args.pp.p[ik];
                alpha = ga.ea[ib];
                beta = p - alpha;
                gamma = ga.ea[ik];
                const double Px = args.pp.px[ib], Py = args.pp.py[ib], Pz = args.pp.pz[ib];
                const double Qx = args.pp.px[ik], Qy = args.pp.py[ik], Qz = args.pp.pz[ik];
                const double ppq = p + q, rs = rsqrt(ppq);
                const double pre = kSRg * args.pp.cut[ib] * args.pp.cut[ik] * rs;
                if (pre < args.prim_cut) {    // primitive cut of twoints.c:109-111
                    work = false;
                } else {
                    sr = kSRg * args.pp.K[ib] * args.pp.K[ik] * rs;
                    pax = Px - ax; pay = Py - ay; paz = Pz - az;
                    qcx = Qx - cx; qcy = Qy - cy; qcz = Qz - cz;
                    pqx = Px - Qx; pqy = Py - Qy; pqz = Pz - Qz;
                    const double T = p * q / ppq * (pqx * pqx + pqy * pqy + pqz * pqz);
                    for (int f = lane; f < 2 * NR; f += TQ)
                        s_rw[f] = rys_eval(NR, f, T, c_rys, args.rys_coef, kRysDegG);
                }
            }
            __syncthreads();
            if (work) {
                const double ppq = p + q;
                for (int j = lane; j < 3 * NR; j += TQ) {
                    const int r = j / 3, dim = j - 3 * r;
                    const double x = s_rw[r], w = s_rw[NR + r];
                    const double f = x / ppq, B00 = 0.5 * f;
                    const double B10 = (0.5 - B00 * q) / p, B01 = (0.5 - B00 * p) / q;
                    const double pa = dim == 0 ? pax : (dim == 1 ? pay : paz);
                    const double qc = dim == 0 ? qcx : (dim == 1 ? qcy : qcz);
                    const double pq = dim == 0 ? pqx : (dim == 1 ? pqy : pqz);
                    grad_vrr(s_G + (size_t)(dim * NR + r) * dm.gsz, dm.l12, dm.l34, dim == 2 ? w * sr : 1.0, B00,
                             B10, B01, pa - q * pq * f, qc + p * pq * f);
                }
            }
            __syncthreads();
            if (work) {
                // transfer, one (direction, entry, root) per lane and step:
                // I = sum_i C(b,i) ab^i sum_k C(d,k) cd^k G[a+b-i][c+d-k]
                const int W = dm.l34 + 1;
                const int njob = 3 * TSZ * NR;
                for (int jb = lane; jb < njob; jb += TQ) {
                    const int r = jb % NR, e = (jb / NR) % TSZ, dim = jb / (NR * TSZ);
                    const int d = e % dm.ed, c = (e / dm.ed) % dm.ec, b = (e / SB) % dm.eb, a = e / SA;
                    if (a + b > dm.l12 || c + d > dm.l34) continue;
                    const double ab = dim == 0 ? abx : (dim == 1 ? aby : abz);
                    const double cd = dim == 0 ? cdx : (dim == 1 ? cdy : cdz);
                    const double *G = s_G + (size_t)(dim * NR + r) * dm.gsz;
                    double sacc = 0.0, abp = 1.0;
                    int bi = 1;
                    for (int i = 0; i <= b; ++i) {
                        const double *Gi = G + (a + b - i) * W + c + d;
                        double t = 0.0, cdp = 1.0;
                        int bk = 1;
                        for (int k = 0; k <= d; ++k) {
                            t = fma(bk * cdp, Gi[-k], t);
                            cdp *= cd;
                            bk = bk * (d - k) / (k + 1);
                        }
                        sacc = fma(bi * abp, t, sacc);
                        abp *= ab;
                        bi = bi * (b - i) / (i + 1);
                    }
                    s_tab[jb] = sacc;
                }
            }
            __syncthreads();
            if (work) {
                const double ta = 2.0 * alpha, tb = 2.0 * beta, tc = 2.0 * gamma;
                for (int c = lane; c < NCART; c += TQ) {
                    const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
                    const int ea = c_cart[dm.la][ia], eb = c_cart[dm.lb][ib], ec = c_cart[dm.lc][ic],
                              ed = c_cart[dm.ld][id];
                    int e0[3];
#pragma unroll
                    for (int dim = 0; dim < 3; ++dim) {
                        const int sh = 4 * dim;
                        e0[dim] = (((ea >> sh) & 15) * dm.eb + ((eb >> sh) & 15)) * dm.ec * dm.ed +
                                  ((ec >> sh) & 15) * dm.ed + ((ed >> sh) & 15);
                    }
                    const double gm = s_gam[c];
#pragma unroll
                    for (int dim = 0; dim < 3; ++dim) {
                        const int sh = 4 * dim;
                        const int xa = (ea >> sh) & 15, xb = (eb >> sh) & 15, xc = (ec >> sh) & 15;
                        const int d1 = dim == 0 ? 1 : 0, d2 = dim == 2 ? 1 : 2;
                        const double *t0 = s_tab + (size_t)dim * TSZ * NR;
                        const double *t1 = s_tab + ((size_t)d1 * TSZ + e0[d1]) * NR;
                        const double *t2 = s_tab + ((size_t)d2 * TSZ + e0[d2]) * NR;
                        // lowered entries are read only when the exponent is positive
                        const int e = e0[dim];
                        const double *pa1 = t0 + (size_t)(e + SA) * NR, *ma1 = t0 + (size_t)(xa > 0 ? e - SA : e) * NR;
                        const double *pb1 = t0 + (size_t)(e + SB) * NR, *mb1 = t0 + (size_t)(xb > 0 ? e - SB : e) * NR;
                        const double *pc1 = t0 + (size_t)(e + SC) * NR, *mc1 = t0 + (size_t)(xc > 0 ? e - SC : e) * NR;
                        double sA = 0.0, sB = 0.0, sC = 0.0;
                        for (int r = 0; r < NR; ++r) {
                            const double o = t1[r] * t2[r];
                            double dA = ta * pa1[r];
                            if (xa > 0) dA = fma(-(double)xa, ma1[r], dA);
                            double dB = tb * pb1[r];
                            if (xb > 0) dB = fma(-(double)xb, mb1[r], dB);
                            double dC = tc * pc1[r];
                            if (xc > 0) dC = fma(-(double)xc, mc1[r], dC);
                            sA = fma(dA, o, sA);
                            sB = fma(dB, o, sB);
                            sC = fma(dC, o, sC);
                        }
                        g[dim] = fma(gm, sA, g[dim]);
                        g[3 + dim] = fma(gm, sB, g[3 + dim]);
                        g[6 + dim] = fma(gm, sC, g[6 + dim]);
                    }
                }
            }
            __syncthreads();
        }
        // team reduction (TQ >= 8: a lane sums at most two of the nine rows);
        // lanes 0..2 then add the x, y, z of the four centres
#pragma unroll
        for (int k = 0; k < 9; ++k) s_red[k * TQ + lane] = g[k];
        __syncthreads();
        double rsum[2] = {0.0, 0.0};
        for (int k = lane, m = 0; k < 9; k += TQ, ++m)
            for (int t = 0; t < TQ; ++t) rsum[m] += s_red[k * TQ + t];
        __syncthreads();
        for (int k = lane, m = 0; k < 9; k += TQ, ++m) s_red[k * TQ] = rsum[m];
        __syncthreads();
        if (active && lane < 3) {
            const double gA = s_red[lane * TQ], gB = s_red[(3 + lane) * TQ], gC = s_red[(6 + lane) * TQ];
            atomicAdd(ga.grad + 3 * ga.ca[u] + lane, gA);
            atomicAdd(ga.grad + 3 * ga.cb[u] + lane, gB);
            atomicAdd(ga.grad + 3 * ga.ca[v] + lane, gC);
            atomicAdd(ga.grad + 3 * ga.cb[v] + lane, -(gA + gB + gC));
        }
        __syncthreads();
    }
}

}  // namespace

size_t eri_grad_smem(int la, int lb, int lc, int ld)
{
    const GradDims d = grad_dims(la, lb, lc, ld);
    return sizeof(double) * (size_t)d.team * d.nteam;
}

cudaError_t launch_eri_grad(const EriArgs &a, const GradArgs &g, cudaStream_t stream, int num_sms)
{
    if (g.la < 0 || g.la > 3 || g.lb < 0 || g.lb > g.la || g.lc < 0 || g.lc > 3 || g.ld < 0 || g.ld > g.lc)
        return cudaErrorInvalidValue;
    const GradDims d = grad_dims(g.la, g.lb, g.lc, g.ld);
    const size_t smem = sizeof(double) * (size_t)d.team * d.nteam;
    static size_t configured = 0;
    if (smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(eri_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    long long blocks = (a.nquart + d.nteam - 1) / d.nteam;
    const long long cap = (long long)num_sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) return cudaSuccess;
    EriArgs b = a;
    b.swap = 0;
    eri_grad_kernel<<<(unsigned)blocks, kBlk, smem, stream>>>(b, g, d);
    return cudaGetLastError();
}

}  // namespace pg
