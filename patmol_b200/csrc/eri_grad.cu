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

#include <mutex>
#include <vector>

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
    int nr, nrp, l12, l34, ea, eb, ec, ed, tsz, gsz, nvalid;
    int tq, nteam, rw, team;   // team: doubles of shared memory per team
    const int4 *desc;          // per component: table entries, exponents, component indices
    const int2 *ent;           // per valid transfer entry: table index, (a, b, c, d)
};

// Host-built index tables of every class (uploaded once per process):
//  desc[c] = {e_x | e_y << 10 | e_z << 20,   1-D table entry of component c per direction
//             exponents (a, b, c of the quartet) per direction, 2 bits each,
//             ia | ib << 4 | ic << 8 | id << 12,   component indices
//             0}
//  ent[k]  = {table index e, a | b << 4 | c << 8 | d << 12} for the entries
//             with a + b <= la + lb + 1 and c + d <= lc + ld + 1.
struct GradTables {
    int4 *desc = nullptr;
    int2 *ent = nullptr;
    long long doff[4][4][4][4], eoff[4][4][4][4];
    int nvalid[4][4][4][4];
    cudaError_t status = cudaSuccess;
};

int cexp_host(int l, int k, int dir)
{
    int n = 0;
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
            if (n == k) return dir == 0 ? lx : (dir == 1 ? ly : l - lx - ly);
            ++n;
        }
    return 0;
}

// one copy per device (the tables hold device addresses)
const GradTables &grad_tables()
{
    static GradTables tabs[64];
    static std::once_flag once[64];
    int dev = 0;
    cudaGetDevice(&dev);
    GradTables &t = tabs[dev & 63];
    std::call_once(once[dev & 63], [&t] {
        std::vector<int4> desc;
        std::vector<int2> ent;
        auto nc = [](int l) { return (l + 1) * (l + 2) / 2; };
        for (int la = 0; la < 4; ++la)
            for (int lb = 0; lb <= la; ++lb)
                for (int lc = 0; lc < 4; ++lc)
                    for (int ld = 0; ld <= lc; ++ld) {
                        const int EB = lb + 2, EC = lc + 2, ED = ld + 1;
                        t.doff[la][lb][lc][ld] = (long long)desc.size();
                        for (int ia = 0; ia < nc(la); ++ia)
                            for (int ib = 0; ib < nc(lb); ++ib)
                                for (int ic = 0; ic < nc(lc); ++ic)
                                    for (int id = 0; id < nc(ld); ++id) {
                                        int e = 0, x = 0;
                                        for (int dim = 0; dim < 3; ++dim) {
                                            const int a = cexp_host(la, ia, dim), b = cexp_host(lb, ib, dim);
                                            const int c = cexp_host(lc, ic, dim), d = cexp_host(ld, id, dim);
                                            e |= (((a * EB + b) * EC + c) * ED + d) << (10 * dim);
                                            x |= (a | b << 2 | c << 4) << (6 * dim);
                                        }
                                        desc.push_back(make_int4(e, x, ia | ib << 4 | ic << 8 | id << 12, 0));
                                    }
                        t.eoff[la][lb][lc][ld] = (long long)ent.size();
                        int nv = 0;
                        for (int a = 0; a < la + 2; ++a)
                            for (int b = 0; b < EB; ++b)
                                for (int c = 0; c < EC; ++c)
                                    for (int d = 0; d < ED; ++d) {
                                        if (a + b > la + lb + 1 || c + d > lc + ld + 1) continue;
                                        ent.push_back(make_int2(((a * EB + b) * EC + c) * ED + d,
                                                                a | b << 4 | c << 8 | d << 12));
                                        ++nv;
                                    }
                        t.nvalid[la][lb][lc][ld] = nv;
                    }
        cudaError_t e = cudaMalloc(&t.desc, sizeof(int4) * desc.size());
        if (e == cudaSuccess) e = cudaMalloc(&t.ent, sizeof(int2) * ent.size());
        if (e == cudaSuccess) e = cudaMemcpy(t.desc, desc.data(), sizeof(int4) * desc.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(t.ent, ent.data(), sizeof(int2) * ent.size(), cudaMemcpyHostToDevice);
        t.status = e;
    });
    return t;
}

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
    d.nrp = d.nr | 1;   // odd root stride: lanes reading neighbouring entries hit different banks
    d.tq = tq_for(d.ncart);
    d.nteam = kBlk / d.tq;
    d.rw = (2 * d.nr + 1) / 2 * 2;
    d.team = (d.rw + 3 * d.nr * d.gsz + 3 * d.nrp * d.tsz + d.ncart + 9 * d.tq + 1) / 2 * 2;
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

    const int TQ = dm.tq, NTEAM = dm.nteam, NR = dm.nr, NRP = dm.nrp, TSZ = dm.tsz;
    const int NCART = dm.ncart;
    const int SA = dm.eb * dm.ec * dm.ed, SB = dm.ec * dm.ed, SC = dm.ed;   // table strides of a, b, c
    const int team = threadIdx.x / TQ, lane = threadIdx.x % TQ;
    double *s_rw = smem + (size_t)team * dm.team;   // nodes [0, NR), weights [NR, 2NR)
    double *s_G = s_rw + dm.rw;                     // [3][NR][gsz] 2-D recursion
    double *s_tab = s_G + 3 * NR * dm.gsz;          // [3][TSZ][NRP]
    double *s_gam = s_tab + 3 * NRP * TSZ;          // [NCART]
    double *s_red = s_gam + NCART;                  // [9][TQ]
    const int n = args.n;
    const double *__restrict__ P = args.D0;
    const double *__restrict__ PB = args.D1;   // set: open shell (P = alpha, PB = beta spin density)

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
                const int ci = __ldg(&dm.desc[c].z);
                const int ia = ci & 15, ib = (ci >> 4) & 15, ic = (ci >> 8) & 15, id = ci >> 12;
                const int i = fa + ia, j = fb + ib, k = fc + ic, l = fd + id;
                const size_t ij = (size_t)i * n + j, kl = (size_t)k * n + l, ik = (size_t)i * n + k,
                             jl = (size_t)j * n + l, il = (size_t)i * n + l, jk = (size_t)j * n + k;
                double g;
                if (!PB) {   // closed shell, half density P
                    g = 2.0 * __ldg(P + ij) * __ldg(P + kl) -
                        0.5 * (__ldg(P + ik) * __ldg(P + jl) + __ldg(P + il) * __ldg(P + jk));
                } else {     // open shell, spin densities Pa = P and Pb
                    const double tij = __ldg(P + ij) + __ldg(PB + ij), tkl = __ldg(P + kl) + __ldg(PB + kl);
                    g = 0.5 * tij * tkl -
                        0.25 * (__ldg(P + ik) * __ldg(P + jl) + __ldg(P + il) * __ldg(P + jk) +
                                __ldg(PB + ik) * __ldg(PB + jl) + __ldg(PB + il) * __ldg(PB + jk));
                }
                s_gam[c] = deg * g * c_norm[dm.la][ia] * c_norm[dm.lb][ib] * c_norm[dm.lc][ic] * c_norm[dm.ld][id];
            }
        }
        int maxp = 1;   // block-uniform; 1 without a reduction when every shell has one primitive
        if (!args.single_prim) {
            if (lane == 0) s_np[team] = active ? npb * npk : 0;
            __syncthreads();
            if (threadIdx.x == 0) {
                int m = 0;
                for (int t = 0; t < NTEAM; ++t) m = max(m, s_np[t]);
                s_maxp = m;
            }
            __syncthreads();
            maxp = s_maxp;
        }
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
                        s_rw[f] = rys_eval(NR, f, T, c_rys, args.rys_coef, kRysDegG, true);
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
                // transfer, one (direction, valid entry) per lane and step, all roots:
                // I = sum_i C(b,i) ab^i sum_k C(d,k) cd^k G[a+b-i][c+d-k]
                const int W = dm.l34 + 1, NV = dm.nvalid;
                for (int jb = lane; jb < 3 * NV; jb += TQ) {
                    const int dim = jb >= 2 * NV ? 2 : (jb >= NV ? 1 : 0), k0 = jb - dim * NV;
                    const int2 en = __ldg(&dm.ent[k0]);
                    const int a = en.y & 15, b = (en.y >> 4) & 15, c = (en.y >> 8) & 15, d = en.y >> 12;
                    const double ab = dim == 0 ? abx : (dim == 1 ? aby : abz);
                    const double cd = dim == 0 ? cdx : (dim == 1 ? cdy : cdz);
                    double cb[5], cdk[4];   // C(b,i) ab^i and C(d,k) cd^k (b <= 4, d <= 3)
                    cb[0] = 1.0;
                    cdk[0] = 1.0;
#pragma unroll
                    for (int i = 1; i < 5; ++i) cb[i] = i <= b ? cb[i - 1] * ab * (double)(b - i + 1) / (double)i : 0.0;
#pragma unroll
                    for (int k = 1; k < 4; ++k) cdk[k] = k <= d ? cdk[k - 1] * cd * (double)(d - k + 1) / (double)k : 0.0;
                    const double *G = s_G + (size_t)dim * NR * dm.gsz + (a + b) * W + c + d;
                    double *out = s_tab + ((size_t)dim * TSZ + en.x) * NRP;
                    for (int r = 0; r < NR; ++r) {
                        const double *Gr = G + r * dm.gsz;
                        double sacc = 0.0;
#pragma unroll
                        for (int i = 0; i < 5; ++i) {
                            if (i > b) break;
                            double t = 0.0;
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                if (k > d) break;
                                t = fma(cdk[k], Gr[-i * W - k], t);
                            }
                            sacc = fma(cb[i], t, sacc);
                        }
                        out[r] = sacc;
                    }
                }
            }
            __syncthreads();
            if (work) {
                const double ta = 2.0 * alpha, tb = 2.0 * beta, tc = 2.0 * gamma;
                for (int c = lane; c < NCART; c += TQ) {
                    const int4 ds = __ldg(&dm.desc[c]);
                    const int e0[3] = {ds.x & 1023, (ds.x >> 10) & 1023, ds.x >> 20};
                    const double gm = s_gam[c];
#pragma unroll
                    for (int dim = 0; dim < 3; ++dim) {
                        const int xs = ds.y >> (6 * dim);
                        const int xa = xs & 3, xb = (xs >> 2) & 3, xc = (xs >> 4) & 3;
                        const int d1 = dim == 0 ? 1 : 0, d2 = dim == 2 ? 1 : 2;
                        const double *t0 = s_tab + (size_t)dim * TSZ * NRP;
                        const double *t1 = s_tab + ((size_t)d1 * TSZ + e0[d1]) * NRP;
                        const double *t2 = s_tab + ((size_t)d2 * TSZ + e0[d2]) * NRP;
                        // lowered entries are read only when the exponent is positive
                        const int e = e0[dim];
                        const double *pa1 = t0 + (size_t)(e + SA) * NRP, *ma1 = t0 + (size_t)(xa > 0 ? e - SA : e) * NRP;
                        const double *pb1 = t0 + (size_t)(e + SB) * NRP, *mb1 = t0 + (size_t)(xb > 0 ? e - SB : e) * NRP;
                        const double *pc1 = t0 + (size_t)(e + SC) * NRP, *mc1 = t0 + (size_t)(xc > 0 ? e - SC : e) * NRP;
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
    GradDims d = grad_dims(g.la, g.lb, g.lc, g.ld);
    const GradTables &t = grad_tables();
    if (t.status != cudaSuccess) return t.status;
    d.desc = t.desc + t.doff[g.la][g.lb][g.lc][g.ld];
    d.ent = t.ent + t.eoff[g.la][g.lb][g.lc][g.ld];
    d.nvalid = t.nvalid[g.la][g.lb][g.lc][g.ld];
    const size_t smem = sizeof(double) * (size_t)d.team * d.nteam;
    // the largest size set so far, per device (the attribute is per device)
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    size_t &conf = configured[dev & 63];
    if (smem > conf) {
        cudaError_t e = cudaFuncSetAttribute(eri_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        conf = smem;
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
