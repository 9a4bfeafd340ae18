// eri_kernel.cuh -- two-electron integrals over contracted Cartesian shell
// quartets by Rys quadrature, fused with their digestion into the
// Coulomb/exchange (G) matrices; the kernel template of one angular-momentum
// class.  Every class is instantiated in its own translation unit.
//
// Algorithm (the same mathematics as twoints.c:23-186 and rys.c:2269-2336):
//   per primitive quartet: p, q, P, Q, T = pq/(p+q)|PQ|^2, n = L/2+1 Rys
//   nodes x_r = t_r^2 and weights w_r; per node and Cartesian direction the
//   2-D recursion G[i][j] (i <= la+lb, j <= lc+ld) from B00, B10, B01, C00,
//   C00'; the binomial transfer to I[a][b][c][d]; the integral of a
//   component quartet is sum_r Ix Iy Iz with w_r and the prefactor
//   2 pi^{5/2} K_ab K_cd / sqrt(p+q) folded into the z factor.
//
// GPU mapping.  A team of TQ = nc*nd threads owns one shell quartet: lane k
// owns ket component k and keeps the integrals of every bra component in
// registers (in compile-time chunks).  Per primitive quartet the team
//   A. evaluates the 2n Chebyshev series of the roots and weights (one
//      lane per series) into shared memory;
//   B. runs the recursion + transfer, one (direction, root) job per lane,
//      into tables laid out [dir][root][ket x-index][bra x-index], so that a
//      lane's slice over the bra x-indices is contiguous;
//   C. accumulates I[ab] += X[ab] Y[ab] Z[ab] over the roots, fully
//      unrolled with compile-time table offsets: each slice entry is loaded
//      once per root and reused by every bra component that shares it.
// Digestion runs from registers: J(cd) and the four exchange partials are
// lane-local dot products against density values staged in shared memory;
// J(ab) and the exchange partials are reduced across the team's lanes
// through shared memory once per quartet.  Density blocks are staged with
// the component factors of basis.c:309-319 folded in, so raw integrals are
// never scaled: each target picks up the factors of its own two components.
//
// Digestion rule (8-fold symmetry with a degeneracy factor instead of the
// reference's per-integral index tests, scfaux.c:446-495): with deg = 8 /
// |symmetry group of the shell quartet| and every component integral v,
//     Jacc(f1,f2) += deg v D(f3,f4)    Jacc(f3,f4) += deg v D(f1,f2)
//     Kacc(f1,f3) += deg v D(f2,f4)    Kacc(f2,f4) += deg v D(f1,f3)
//     Kacc(f1,f4) += deg v D(f2,f3)    Kacc(f2,f3) += deg v D(f1,f4)
// gives J = (Jacc + Jacc^T)/4 and K = (Kacc + Kacc^T)/8; every target adds
// once per quartet into the n x n accumulator (L2 resident) through acc_add:
// exact fixed-point integer adds (order-independent, so G is bitwise
// reproducible) or, with det = 0, FP64 atomics.
#pragma once
#include "eri.cuh"

namespace pg {

// defined in eri.cu (relocatable device code)
extern __constant__ RysConst c_rys;
extern __constant__ int c_cart[4][10];
extern __constant__ double c_norm[4][10];

constexpr double kSR = 34.98683665524972497;   // 2 pi^(5/2)
constexpr int kRysDeg = 11;

constexpr int binom(int n, int k)
{
    int r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// Cartesian exponent (dir 0/1/2 = x/y/z) of component k of angular
// momentum l, in the order of basis.c:294-308.
constexpr int cexp(int l, int k, int dir)
{
    int n = 0;
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
            if (n == k) return dir == 0 ? lx : (dir == 1 ? ly : l - lx - ly);
            ++n;
        }
    return 0;
}

template <int LA, int LB, int LC, int LD, int NDEN>
struct Shape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND, NCART = NAB * NCD;
    static constexpr int L12 = LA + LB, L34 = LC + LD;
    static constexpr int NR = (L12 + L34) / 2 + 1;
    static constexpr int TAB = (LA + 1) * (LB + 1), TCD = (LC + 1) * (LD + 1);
    static constexpr int TSZ = TAB * TCD;
    static constexpr int MAXACC = NDEN == 1 ? 36 : 20;
    static constexpr int NCH = (NAB + MAXACC - 1) / MAXACC;   // bra chunks (<= 5)
    static constexpr int CH = (NAB + NCH - 1) / NCH;           // bra components per chunk
    static constexpr int TQ = NCD;                              // lanes per quartet
    // staged density blocks per set: D(ab), D(bd), D(bc), D(ad), D(ac)
    static constexpr int OBD = NAB, OBC = OBD + NB * ND, OAD = OBC + NB * NC, OAC = OAD + NA * ND;
    static constexpr int NDB = OAC + NA * NC;
    static constexpr int PS = 2 * NA + 2 * NB;                  // exchange partials per lane and set
    static constexpr int NPART = NCD * PS * NDEN;
    static constexpr int NW = NCD > 1 ? NCART : 0;              // J(ab) partials
    static constexpr int REGION = (3 * NR * TSZ > NW + NPART) ? 3 * NR * TSZ : NW + NPART;
    static constexpr int SM_TEAM = 2 * NR + NDB * NDEN + REGION;
    static constexpr int NT0 = (256 / TQ) > 0 ? 256 / TQ : 1;
    static constexpr int NT1 = (NT0 * SM_TEAM * 8 > 96 * 1024) ? ((96 * 1024) / (SM_TEAM * 8)) : NT0;
    static constexpr int NTEAM = NT1 > 0 ? NT1 : 1;
    static constexpr int BLK = ((NTEAM * TQ + 31) / 32) * 32;
    static constexpr size_t SMEM = sizeof(double) * (size_t)SM_TEAM * NTEAM;
    // resident blocks requested from the register allocator: at most 128
    // registers a thread, so latency is hidden by occupancy (measured: 96
    // spills too much, 255 leaves 8 warps an SM)
    static constexpr int MINB = (65536 / (BLK * 128)) > 0 ? 65536 / (BLK * 128) : 1;
};

// 2-D recursion and binomial transfer for one root and one direction;
// writes I[a][b][c][d] to tab[(c(LD+1)+d) * TAB + a(LB+1)+b], for every c
// or (csel >= 0, a constant after unrolling at the call) only c = csel.
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void vrr_hrr(R *__restrict__ tab, R g00, R B00, R B10, R B01, R C, R Cp, R ab, R cd,
                                        int csel = -1)
{
    constexpr int L12 = LA + LB, L34 = LC + LD, TAB = (LA + 1) * (LB + 1);
    R G[L12 + 1][L34 + 1];
    G[0][0] = g00;
    if (L12 > 0) G[1][0] = C * g00;
#pragma unroll
    for (int i = 1; i < L12; ++i) G[i + 1][0] = i * B10 * G[i - 1][0] + C * G[i][0];
#pragma unroll
    for (int j = 0; j < L34; ++j) {
#pragma unroll
        for (int i = 0; i <= L12; ++i) {
            R v = Cp * G[i][j];
            if (j > 0) v = fma(R(j) * B01, G[i][j - 1], v);
            if (i > 0) v = fma(R(i) * B00, G[i - 1][j], v);
            G[i][j + 1] = v;
        }
    }
    R cdp[LD + 1], abp[LB + 1];
    cdp[0] = R(1);
#pragma unroll
    for (int k = 1; k <= LD; ++k) cdp[k] = cdp[k - 1] * cd;
    abp[0] = R(1);
#pragma unroll
    for (int k = 1; k <= LB; ++k) abp[k] = abp[k - 1] * ab;
#pragma unroll
    for (int c = 0; c <= LC; ++c)
#pragma unroll
        for (int d = 0; d <= LD; ++d) {
            if (csel >= 0 && c != csel) continue;
            // ket transfer for every bra index: H[i] = sum_k C(d,k) cd^k G[i][c+d-k]
            R H[L12 + 1];
#pragma unroll
            for (int i = 0; i <= L12; ++i) {
                R t = R(0);
#pragma unroll
                for (int k = 0; k <= d; ++k) t = fma(R(binom(d, k)) * cdp[k], G[i][c + d - k], t);
                H[i] = t;
            }
#pragma unroll
            for (int a = 0; a <= LA; ++a)
#pragma unroll
                for (int b = 0; b <= LB; ++b) {
                    R s = R(0);
#pragma unroll
                    for (int i = 0; i <= b; ++i) s = fma(R(binom(b, i)) * abp[i], H[a + b - i], s);
                    tab[(c * (LD + 1) + d) * TAB + a * (LB + 1) + b] = s;
                }
        }
}

// acc[j] += sum_r X Y Z for bra components CH0 .. CH0+CHN-1 (compile time);
// X, Y, Z point at this lane's slices of root 0, RSTRIDE doubles per root.
template <int LA, int LB, int NR, int RSTRIDE, int CH0, int CHN, typename R>
__device__ __forceinline__ void assemble(R (&acc)[CHN], const R *__restrict__ X, const R *__restrict__ Y,
                                         const R *__restrict__ Z)
{
    constexpr int NB = ncart(LB), NAB = ncart(LA) * ncart(LB);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
#pragma unroll
        for (int j = 0; j < CHN; ++j) {
            const int ab = CH0 + j;
            if (ab < NAB) {
                const int ia = ab / NB, ib = ab % NB;
                const int ox = cexp(LA, ia, 0) * (LB + 1) + cexp(LB, ib, 0);
                const int oy = cexp(LA, ia, 1) * (LB + 1) + cexp(LB, ib, 1);
                const int oz = cexp(LA, ia, 2) * (LB + 1) + cexp(LB, ib, 2);
                acc[j] = fma(X[r * RSTRIDE + ox] * Y[r * RSTRIDE + oy], Z[r * RSTRIDE + oz], acc[j]);
            }
        }
    }
}

// R: arithmetic type of the recursion, tables and integrals (float: the
// mixed-precision form -- roots, weights, prefactors and every digestion
// product and J/K sum stay FP64).
template <int LA, int LB, int LC, int LD, int NDEN, typename R = double>
__global__ void __launch_bounds__(Shape<LA, LB, LC, LD, NDEN>::BLK, Shape<LA, LB, LC, LD, NDEN>::MINB)
eri_class_kernel(const EriArgs args)
{
    using S = Shape<LA, LB, LC, LD, NDEN>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NAB = S::NAB, NCD = S::NCD;
    constexpr int NR = S::NR, TAB = S::TAB, TSZ = S::TSZ, TQ = S::TQ, NTEAM = S::NTEAM;
    constexpr int NCH = S::NCH, CH = S::CH, NDB = S::NDB, PS = S::PS;
    extern __shared__ double smem[];
    __shared__ int s_np[NTEAM];
    __shared__ int s_maxp;

    const int team = threadIdx.x / TQ, lane = threadIdx.x - team * TQ;
    const bool in_team = team < NTEAM;
    double *s_rw = smem + (in_team ? team : 0) * S::SM_TEAM;   // nodes [0, NR), weights [NR, 2NR)
    double *s_db = s_rw + 2 * NR;                              // NDEN staged density sets
    double *s_tab = s_db + NDB * NDEN;                         // tables; later W and partials
    double *s_w = s_tab;                                       // [NAB][NCD]
    double *s_part = s_tab + S::NW;                            // [NDEN][NCD][PS]

    // this lane's ket component
    const int ic = in_team ? lane / ND : 0, id = in_team ? lane - (lane / ND) * ND : 0;
    const int ecx = c_cart[LC][ic], edx = c_cart[LD][id];
    const int tcdx = (ecx & 15) * (LD + 1) + (edx & 15);
    const int tcdy = ((ecx >> 4) & 15) * (LD + 1) + ((edx >> 4) & 15);
    const int tcdz = (ecx >> 8) * (LD + 1) + (edx >> 8);
    const double nfk = c_norm[LC][ic] * c_norm[LD][id];
    const int mode = args.mode;
    const int n = args.n;
    const long long nq = eri_work_count(args), q0 = eri_work_first(args, nq);

    for (long long base = (long long)blockIdx.x * NTEAM; base < nq; base += (long long)gridDim.x * NTEAM) {
        const long long qi = base + team;
        int u = 0, v = 0, npb = 0, npk = 0, pb0 = 0, pk0 = 0;
        const bool active = in_team && qi < nq && eri_quartet_at(args, q0 + qi, u, v);
        double ax = 0, ay = 0, az = 0, abx = 0, aby = 0, abz = 0;
        double cx = 0, cy = 0, cz = 0, cdx = 0, cdy = 0, cdz = 0;
        int fa = 0, fb = 0, fc = 0, fd = 0;
        if (active) {
            npb = args.pr.pnum[u];
            npk = args.pr.pnum[v];
            pb0 = args.pr.pstart[u];
            pk0 = args.pr.pstart[v];
            ax = args.pr.ax[u]; ay = args.pr.ay[u]; az = args.pr.az[u];
            abx = args.pr.abx[u]; aby = args.pr.aby[u]; abz = args.pr.abz[u];
            cx = args.pr.ax[v]; cy = args.pr.ay[v]; cz = args.pr.az[v];
            cdx = args.pr.abx[v]; cdy = args.pr.aby[v]; cdz = args.pr.abz[v];
            fa = args.pr.fa[u]; fb = args.pr.fb[u]; fc = args.pr.fa[v]; fd = args.pr.fb[v];
            if (mode != MODE_EXPORT) {
                // stage the density blocks, component factors folded in
#pragma unroll
                for (int s = 0; s < NDEN; ++s) {
                    const double *D = s == 0 ? args.D0 : args.D1;
                    double *db = s_db + s * NDB;
                    for (int t = lane; t < NDB; t += TQ) {
                        int r0, c0, lr, lc2, ir, icn;
                        if (t < S::OBD) {
                            ir = t / NB; icn = t - ir * NB; r0 = fa; c0 = fb; lr = LA; lc2 = LB;
                        } else if (t < S::OBC) {
                            const int tt = t - S::OBD; ir = tt / ND; icn = tt - ir * ND; r0 = fb; c0 = fd; lr = LB; lc2 = LD;
                        } else if (t < S::OAD) {
                            const int tt = t - S::OBC; ir = tt / NC; icn = tt - ir * NC; r0 = fb; c0 = fc; lr = LB; lc2 = LC;
                        } else if (t < S::OAC) {
                            const int tt = t - S::OAD; ir = tt / ND; icn = tt - ir * ND; r0 = fa; c0 = fd; lr = LA; lc2 = LD;
                        } else {
                            const int tt = t - S::OAC; ir = tt / NC; icn = tt - ir * NC; r0 = fa; c0 = fc; lr = LA; lc2 = LC;
                        }
                        db[t] = __ldg(D + (size_t)(r0 + ir) * n + c0 + icn) * c_norm[lr][ir] * c_norm[lc2][icn];
                    }
                }
            }
        }
        // primitive-quartet count of the block (block-uniform for the barriers
        // inside the loop); with one primitive per shell it is 1 without a
        // block reduction
        int maxp = 1;
        if (!args.single_prim) {
            if (in_team && lane == 0) s_np[team] = active ? npb * npk : 0;
            __syncthreads();
            if (threadIdx.x == 0) {
                int m = 0;
                for (int t = 0; t < NTEAM; ++t) m = max(m, s_np[t]);
                s_maxp = m;
            }
            __syncthreads();
            maxp = s_maxp;
        }

        // integrals of every bra component for this lane's ket component
        R acc[NCH][CH];
#pragma unroll
        for (int c = 0; c < NCH; ++c)
#pragma unroll
            for (int j = 0; j < CH; ++j) acc[c][j] = R(0);

        for (int ip = 0; ip < maxp; ++ip) {
            bool work = active && ip < npb * npk;
            double p = 1, q = 1, sr = 0, pax = 0, pay = 0, paz = 0, qcx = 0, qcy = 0, qcz = 0;
            double pqx = 0, pqy = 0, pqz = 0;
            if (work) {
                const int ib = pb0 + ip / npk, ik = pk0 + ip % npk;
                p = args.pp.p[ib];
                q = args.pp.p[ik];
                const double Px = args.pp.px[ib], Py = args.pp.py[ib], Pz = args.pp.pz[ib];
                const double Qx = args.pp.px[ik], Qy = args.pp.py[ik], Qz = args.pp.pz[ik];
                const double ppq = p + q, rs = rsqrt(ppq);
                const double pre = kSR * args.pp.cut[ib] * args.pp.cut[ik] * rs;
                if (pre < args.prim_cut) {    // primitive cut of twoints.c:109-111
                    work = false;
                } else {
                    sr = kSR * args.pp.K[ib] * args.pp.K[ik] * rs;
                    pax = Px - ax; pay = Py - ay; paz = Pz - az;
                    qcx = Qx - cx; qcy = Qy - cy; qcz = Qz - cz;
                    pqx = Px - Qx; pqy = Py - Qy; pqz = Pz - Qz;
                    const double T = p * q / ppq * (pqx * pqx + pqy * pqy + pqz * pqz);
                    for (int f = lane; f < 2 * NR; f += TQ)
                        s_rw[f] = rys_eval(NR, f, T, c_rys, args.rys_coef, kRysDeg, true);
                }
            }
            __syncthreads();
            if (work) {
                const double ppq = p + q;
                // one job per (direction, root); when the team has lanes to
                // spare, one per (direction, root, ket x-index c) instead, each
                // redoing the short 2-D recursion and transferring one c
                constexpr int NSPLIT = (LC > 0 && 3 * NR * (LC + 1) <= TQ) ? LC + 1 : 1;
                for (int j = lane; j < 3 * NR * NSPLIT; j += TQ) {
                    const int cs = j / (3 * NR), jj = j - cs * (3 * NR);
                    const int dim = jj / NR, r = jj - dim * NR;
                    const double x = s_rw[r], w = s_rw[NR + r];
                    const double f = x / ppq, B00 = 0.5 * f;
                    const double B10 = (0.5 - B00 * q) / p, B01 = (0.5 - B00 * p) / q;
                    const double pa = dim == 0 ? pax : (dim == 1 ? pay : paz);
                    const double qc = dim == 0 ? qcx : (dim == 1 ? qcy : qcz);
                    const double pq = dim == 0 ? pqx : (dim == 1 ? pqy : pqz);
                    const double ab = dim == 0 ? abx : (dim == 1 ? aby : abz);
                    const double cd = dim == 0 ? cdx : (dim == 1 ? cdy : cdz);
                    R *tab = reinterpret_cast<R *>(s_tab) + (dim * NR + r) * TSZ;
                    if constexpr (NSPLIT == 1) {
                        vrr_hrr<LA, LB, LC, LD, R>(tab, R(dim == 2 ? w * sr : 1.0), R(B00), R(B10), R(B01),
                                                   R(pa - q * pq * f), R(qc + p * pq * f), R(ab), R(cd));
                    } else {
#pragma unroll
                        for (int c0 = 0; c0 < NSPLIT; ++c0)
                            if (c0 == cs)
                                vrr_hrr<LA, LB, LC, LD, R>(tab, R(dim == 2 ? w * sr : 1.0), R(B00), R(B10), R(B01),
                                                           R(pa - q * pq * f), R(qc + p * pq * f), R(ab), R(cd),
                                                           c0);
                    }
                }
            }
            __syncthreads();
            if (work) {
                const R *tb = reinterpret_cast<const R *>(s_tab);
                const R *X = tb + tcdx * TAB;
                const R *Y = tb + NR * TSZ + tcdy * TAB;
                const R *Z = tb + 2 * NR * TSZ + tcdz * TAB;
                assemble<LA, LB, NR, TSZ, 0, CH>(acc[0], X, Y, Z);
                if constexpr (NCH > 1) assemble<LA, LB, NR, TSZ, CH, CH>(acc[1], X, Y, Z);
                if constexpr (NCH > 2) assemble<LA, LB, NR, TSZ, 2 * CH, CH>(acc[2], X, Y, Z);
                if constexpr (NCH > 3) assemble<LA, LB, NR, TSZ, 3 * CH, CH>(acc[3], X, Y, Z);
                if constexpr (NCH > 4) assemble<LA, LB, NR, TSZ, 4 * CH, CH>(acc[4], X, Y, Z);
            }
            __syncthreads();
        }

        // ------------------------------------------------------ export
        if (mode == MODE_EXPORT) {
            if (active) {
                double *o = args.out + args.out_off[qi];
#pragma unroll
                for (int c = 0; c < NCH; ++c)
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int ab = c * CH + j;
                        if (ab < NAB) {
                            // the caller's orientation: (quart.x pair | quart.y pair)
                            const size_t oi = args.swap ? (size_t)lane * NAB + ab : (size_t)ab * NCD + lane;
                            o[oi] = (double)acc[c][j] * nfk * c_norm[LA][ab / NB] * c_norm[LB][ab % NB];
                        }
                    }
            }
            __syncthreads();
            continue;
        }

        // ---------------------------------------------------- digestion
        const bool sab = active && args.pr.sa[u] == args.pr.sb[u];
        const bool scd = active && args.pr.sa[v] == args.pr.sb[v];
        const double deg = (sab ? 1.0 : 2.0) * (scd ? 1.0 : 2.0) * (u == v ? 1.0 : 2.0);
        const double sJ = mode == MODE_RHF ? 0.5 * deg : 0.25 * deg;
        const double sK = 0.125 * deg;
        if (active) {
            // D(cd) of this lane (Coulomb density: the sum of the sets), factors folded in
            double Dcd = __ldg(args.D0 + (size_t)(fc + ic) * n + fd + id);
            if (NDEN == 2) Dcd += __ldg(args.D1 + (size_t)(fc + ic) * n + fd + id);
            Dcd *= nfk;
            double jcd = 0.0;
            double Pac[NDEN][NA], Pad[NDEN][NA], Pbc[NDEN][NB], Pbd[NDEN][NB];
#pragma unroll
            for (int s = 0; s < NDEN; ++s) {
#pragma unroll
                for (int a = 0; a < NA; ++a) { Pac[s][a] = 0.0; Pad[s][a] = 0.0; }
#pragma unroll
                for (int b = 0; b < NB; ++b) { Pbc[s][b] = 0.0; Pbd[s][b] = 0.0; }
            }
#pragma unroll
            for (int c = 0; c < NCH; ++c)
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int ab = c * CH + j;
                    if (ab < NAB) {
                        const int ia = ab / NB, ib = ab % NB;
                        const double I = (double)acc[c][j];
                        double dab = s_db[ab];
                        if (NDEN == 2) dab += s_db[NDB + ab];
                        jcd = fma(I, dab, jcd);
                        if (NCD > 1) s_w[ab * NCD + lane] = I * Dcd;
#pragma unroll
                        for (int s = 0; s < NDEN; ++s) {
                            const double *db = s_db + s * NDB;
                            Pac[s][ia] = fma(I, db[S::OBD + ib * ND + id], Pac[s][ia]);
                            Pad[s][ia] = fma(I, db[S::OBC + ib * NC + ic], Pad[s][ia]);
                            Pbc[s][ib] = fma(I, db[S::OAD + ia * ND + id], Pbc[s][ib]);
                            Pbd[s][ib] = fma(I, db[S::OAC + ia * NC + ic], Pbd[s][ib]);
                        }
                    }
                }
            // J(cd): complete in this lane
            {
                const double o = sJ * jcd * nfk;
                const size_t idx = (size_t)(fc + ic) * n + fd + id;
                acc_add(args.A0, idx, o, args.det, args.err);
                if (NDEN == 2) acc_add(args.A1, idx, o, args.det, args.err);
            }
            if constexpr (NCD == 1) {
                // a single ket component: J(ab) and the exchange targets are lane-local
#pragma unroll
                for (int c = 0; c < NCH; ++c)
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int ab = c * CH + j;
                        if (ab < NAB) {
                            const int ia = ab / NB, ib = ab % NB;
                            const double o = sJ * (double)acc[c][j] * Dcd * c_norm[LA][ia] * c_norm[LB][ib];
                            const size_t idx = (size_t)(fa + ia) * n + fb + ib;
                            acc_add(args.A0, idx, o, args.det, args.err);
                            if (NDEN == 2) acc_add(args.A1, idx, o, args.det, args.err);
                        }
                    }
#pragma unroll
                for (int s = 0; s < NDEN; ++s) {
                    double *A = mode == MODE_JK ? args.A1 : (s == 0 ? args.A0 : args.A1);
                    const double sg = mode == MODE_JK ? sK : -sK;
#pragma unroll
                    for (int a = 0; a < NA; ++a) {
                        acc_add(A, (size_t)(fa + a) * n + fc, sg * Pac[s][a] * c_norm[LA][a], args.det, args.err);
                        acc_add(A, (size_t)(fa + a) * n + fd, sg * Pad[s][a] * c_norm[LA][a], args.det, args.err);
                    }
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        acc_add(A, (size_t)(fb + b) * n + fc, sg * Pbc[s][b] * c_norm[LB][b], args.det, args.err);
                        acc_add(A, (size_t)(fb + b) * n + fd, sg * Pbd[s][b] * c_norm[LB][b], args.det, args.err);
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < NDEN; ++s) {
                    double *pp = s_part + ((size_t)s * NCD + lane) * PS;
#pragma unroll
                    for (int a = 0; a < NA; ++a) { pp[a] = Pac[s][a]; pp[NA + a] = Pad[s][a]; }
#pragma unroll
                    for (int b = 0; b < NB; ++b) { pp[2 * NA + b] = Pbc[s][b]; pp[2 * NA + NB + b] = Pbd[s][b]; }
                }
            }
        }
        if constexpr (NCD > 1) {
            __syncthreads();
            if (active) {
                // cross-lane reductions, one target per lane
                constexpr int T0 = NAB, T1 = T0 + NA * NC, T2 = T1 + NA * ND, T3 = T2 + NB * NC,
                              T4 = T3 + NB * ND;
                for (int t = lane; t < T4; t += TQ) {
                    if (t < T0) {
                        const int ia = t / NB, ib = t - (t / NB) * NB;
                        double s = 0.0;
#pragma unroll 4
                        for (int k = 0; k < NCD; ++k) s += s_w[t * NCD + k];
                        const double o = sJ * s * c_norm[LA][ia] * c_norm[LB][ib];
                        const size_t idx = (size_t)(fa + ia) * n + fb + ib;
                        acc_add(args.A0, idx, o, args.det, args.err);
                        if (NDEN == 2) acc_add(args.A1, idx, o, args.det, args.err);
                        continue;
                    }
                    int row, col, base2, stride, cnt, off, lr, lc2, ir, icl;
                    if (t < T1) {          // K(a,c) = sum_d Pac[(c,d)][a]
                        const int tt = t - T0; ir = tt / NC; icl = tt - ir * NC;
                        row = fa + ir; col = fc + icl; base2 = icl * ND; stride = 1; cnt = ND; off = ir;
                        lr = LA; lc2 = LC;
                    } else if (t < T2) {   // K(a,d) = sum_c Pad[(c,d)][a]
                        const int tt = t - T1; ir = tt / ND; icl = tt - ir * ND;
                        row = fa + ir; col = fd + icl; base2 = icl; stride = ND; cnt = NC; off = NA + ir;
                        lr = LA; lc2 = LD;
                    } else if (t < T3) {   // K(b,c) = sum_d Pbc[(c,d)][b]
                        const int tt = t - T2; ir = tt / NC; icl = tt - ir * NC;
                        row = fb + ir; col = fc + icl; base2 = icl * ND; stride = 1; cnt = ND; off = 2 * NA + ir;
                        lr = LB; lc2 = LC;
                    } else {               // K(b,d) = sum_c Pbd[(c,d)][b]
                        const int tt = t - T3; ir = tt / ND; icl = tt - ir * ND;
                        row = fb + ir; col = fd + icl; base2 = icl; stride = ND; cnt = NC; off = 2 * NA + NB + ir;
                        lr = LB; lc2 = LD;
                    }
                    const double f = sK * c_norm[lr][ir] * c_norm[lc2][icl];
                    const size_t idx = (size_t)row * n + col;
#pragma unroll
                    for (int s = 0; s < NDEN; ++s) {
                        double sum = 0.0;
                        for (int k = 0; k < cnt; ++k) sum += s_part[((size_t)s * NCD + base2 + k * stride) * PS + off];
                        if (mode == MODE_JK) acc_add(args.A1, idx, f * sum, args.det, args.err);
                        else acc_add(s == 0 ? args.A0 : args.A1, idx, -f * sum, args.det, args.err);
                    }
                }
            }
        }
        // With more than one lane, the barrier before the cross-lane phase
        // already separates every read of the staged densities from the next
        // quartet's staging, and the next quartet writes the tables that
        // phase reads only after its roots barrier.  A one-lane team's
        // digestion reads the staged densities directly, so it keeps this one.
        if constexpr (NCD == 1) __syncthreads();
    }
}

template <int LA, int LB, int LC, int LD, int NDEN, typename R = double>
cudaError_t launch_one(const EriArgs &a, cudaStream_t stream, int num_sms)
{
    using S = Shape<LA, LB, LC, LD, NDEN>;
    static unsigned long long configured = 0;   // per device: the attribute is per device
    if (first_on_device(&configured)) {
        cudaError_t e = cudaFuncSetAttribute(eri_class_kernel<LA, LB, LC, LD, NDEN, R>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return e;
    }
    static int resident[64] = {};
    long long blocks = (a.nquart + S::NTEAM - 1) / S::NTEAM;
    const long long cap = (long long)num_sms *
        resident_blocks((const void *)eri_class_kernel<LA, LB, LC, LD, NDEN, R>, S::BLK, S::SMEM, resident);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) return cudaSuccess;
    eri_class_kernel<LA, LB, LC, LD, NDEN, R><<<(unsigned)blocks, S::BLK, S::SMEM, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace pg
