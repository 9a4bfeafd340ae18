// eri_smem.cuh -- the shared-memory team variant of the shell-quartet
// kernel: a team of TQ threads (1..128 by class size) owns one quartet, the
// 1-D Rys tables and the whole integral block live in shared memory, and each
// J/K target is a dot product over the block computed by one lane.  Same
// mathematics and digestion rule as eri_kernel.cuh (which see); the
// autotuner picks, per class, whichever variant runs fastest.
//
// The arithmetic type R of the recursion, tables and integrals is a template
// parameter: R = float gives the mixed-precision path for quartets whose
// Schwarz bound is small -- roots and weights, prefactors and T are still
// FP64, and every digestion product and J/K sum is formed in FP64.
#pragma once
#include "eri_kernel.cuh"

namespace pg {


constexpr int pick_tq(int ncart_total)
{
    return ncart_total <= 12 ? 1
         : ncart_total <= 40 ? 2
         : ncart_total <= 120 ? 4
         : ncart_total <= 300 ? 8
         : ncart_total <= 700 ? 16
         : ncart_total <= 1500 ? 32
         : ncart_total <= 3000 ? 64 : 128;
}

template <int LA, int LB, int LC, int LD, typename R>
struct SmemShape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NCART = NA * NB * NC * ND;
    static constexpr int L12 = LA + LB, L34 = LC + LD;
    static constexpr int NR = (L12 + L34) / 2 + 1;
    static constexpr int TSZ = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    static constexpr int TQ = pick_tq(NCART);
    static constexpr int BLK = 128;
    static constexpr int NTEAM = BLK / TQ;
    // bytes per team: roots and weights (FP64), tables and integrals (R)
    static constexpr int TEAM_BYTES = ((16 * NR + (int)sizeof(R) * (3 * NR * TSZ + NCART)) + 15) / 16 * 16;
    static constexpr size_t SMEM = (size_t)TEAM_BYTES * NTEAM;
    // blocks an SM can hold by shared memory (228 KB an SM, 1 KB reserved a
    // block), and the blocks per SM the occupancy-hinted form asks of the
    // register allocator: up to 4 (16 warps, at most 128 registers a thread)
    static constexpr int SMEM_BLOCKS = (int)((228 * 1024) / (SMEM + 1024));
    static constexpr int OCC = SMEM_BLOCKS >= 4 ? 4 : SMEM_BLOCKS;
    // the hinted form exists where it lowers the register cap below the 255
    // of the plain form, i.e. where shared memory leaves room for 3+ blocks
    static constexpr bool HAS_OCC = OCC >= 3;
};

// 2-D recursion (rys.c:2269-2293 in the reference) and binomial transfer
// (rys.c:2295-2336) for one root and one Cartesian direction; writes
// I[a][b][c][d] into tab[idx * NR] with idx = ((a(LB+1)+b)(LC+1)+c)(LD+1)+d.
template <int LA, int LB, int LC, int LD, int NR, typename R>
__device__ __forceinline__ void vrr_hrr_smem(R *__restrict__ tab, R g00, R B00, R B10, R B01, R C, R Cp, R ab,
                                             R cd)
{
    constexpr int L12 = LA + LB, L34 = LC + LD;
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
    // ket transfer H[i][c][d] = sum_k C(d,k) cd^k G[i][c+d-k], then bra
    R cdp[LD + 1], abp[LB + 1];
    cdp[0] = R(1);
#pragma unroll
    for (int k = 1; k <= LD; ++k) cdp[k] = cdp[k - 1] * cd;
    abp[0] = R(1);
#pragma unroll
    for (int k = 1; k <= LB; ++k) abp[k] = abp[k - 1] * ab;
#pragma unroll
    for (int a = 0; a <= LA; ++a)
#pragma unroll
        for (int b = 0; b <= LB; ++b)
#pragma unroll
            for (int c = 0; c <= LC; ++c)
#pragma unroll
                for (int d = 0; d <= LD; ++d) {
                    R s = R(0);
#pragma unroll
                    for (int i = 0; i <= b; ++i) {
                        R t = R(0);
#pragma unroll
                        for (int k = 0; k <= d; ++k) t = fma(R(binom(d, k)) * cdp[k], G[a + b - i][c + d - k], t);
                        s = fma(R(binom(b, i)) * abp[i], t, s);
                    }
                    const int idx = ((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d;
                    tab[idx * NR] = s;
                }
}

// MINB > 1: the occupancy-hinted form, whose register allocation is capped so
// that MINB blocks of 128 threads fit an SM (the autotuner times it beside
// the plain form, MINB = 1).
template <int LA, int LB, int LC, int LD, typename R, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) eri_smem_kernel(const EriArgs args)
{
    using S = SmemShape<LA, LB, LC, LD, R>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NCART = S::NCART;
    constexpr int NR = S::NR, TSZ = S::TSZ, TQ = S::TQ, NTEAM = S::NTEAM;
    extern __shared__ double smem[];
    __shared__ int s_np[NTEAM];
    __shared__ int s_maxp;

    const int team = threadIdx.x / TQ, lane = threadIdx.x % TQ;
    double *s_rw = reinterpret_cast<double *>(reinterpret_cast<char *>(smem) + team * S::TEAM_BYTES);  // nodes, weights
    R *s_tab = reinterpret_cast<R *>(s_rw + 2 * NR);   // [3][TSZ][NR]
    R *s_out = s_tab + 3 * NR * TSZ;                   // [NCART]

    const long long nq = eri_work_count(args), q0 = eri_work_first(args, nq);
    for (long long base = (long long)blockIdx.x * NTEAM; base < nq; base += (long long)gridDim.x * NTEAM) {
        const long long qi = base + team;
        int u = 0, v = 0, npb = 0, npk = 0, pb0 = 0, pk0 = 0;
        const bool active = qi < nq && eri_quartet_at(args, q0 + qi, u, v);
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
        }
        for (int c = lane; c < NCART; c += TQ) s_out[c] = R(0);
        int maxp = 1;   // block-uniform; 1 without a reduction when every shell has one primitive
        if (!args.single_prim) {
            if (lane == 0) s_np[team] = npb * npk;
            __syncthreads();
            if (threadIdx.x == 0) {
                int m = 0;
                for (int t = 0; t < NTEAM; ++t) m = max(m, s_np[t]);
                s_maxp = m;
            }
            __syncthreads();
            maxp = s_maxp;
        }

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
                for (int j = lane; j < 3 * NR; j += TQ) {
                    const int r = j / 3, dim = j - 3 * r;
                    const double x = s_rw[r], w = s_rw[NR + r];
                    const double f = x / ppq, B00 = 0.5 * f;
                    const double B10 = (0.5 - B00 * q) / p, B01 = (0.5 - B00 * p) / q;
                    const double pa = dim == 0 ? pax : (dim == 1 ? pay : paz);
                    const double qc = dim == 0 ? qcx : (dim == 1 ? qcy : qcz);
                    const double pq = dim == 0 ? pqx : (dim == 1 ? pqy : pqz);
                    const double ab = dim == 0 ? abx : (dim == 1 ? aby : abz);
                    const double cd = dim == 0 ? cdx : (dim == 1 ? cdy : cdz);
                    vrr_hrr_smem<LA, LB, LC, LD, NR, R>(s_tab + dim * TSZ * NR + r, R(dim == 2 ? w * sr : 1.0), R(B00),
                                                        R(B10), R(B01), R(pa - q * pq * f), R(qc + p * pq * f), R(ab),
                                                        R(cd));
                }
            }
            __syncthreads();
            if (work) {
                for (int c = lane; c < NCART; c += TQ) {
                    const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
                    const int ea = c_cart[LA][ia], eb = c_cart[LB][ib], ec = c_cart[LC][ic], ed = c_cart[LD][id];
                    const int ix = ((((ea & 15) * (LB + 1) + (eb & 15)) * (LC + 1) + (ec & 15)) * (LD + 1) + (ed & 15));
                    const int iy = (((((ea >> 4) & 15) * (LB + 1) + ((eb >> 4) & 15)) * (LC + 1) + ((ec >> 4) & 15)) *
                                        (LD + 1) + ((ed >> 4) & 15));
                    const int iz = ((((ea >> 8) * (LB + 1) + (eb >> 8)) * (LC + 1) + (ec >> 8)) * (LD + 1) + (ed >> 8));
                    const R *tx = s_tab + ix * NR, *ty = s_tab + (TSZ + iy) * NR, *tz = s_tab + (2 * TSZ + iz) * NR;
                    R s = R(0);
#pragma unroll
                    for (int r = 0; r < NR; ++r) s = fma(tx[r] * ty[r], tz[r], s);
                    s_out[c] += s;
                }
            }
            __syncthreads();
        }

        // ------------------------------------------------ digestion / export
        if (active) {
            // component factors (basis.c:309-319)
            for (int c = lane; c < NCART; c += TQ) {
                const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
                s_out[c] *= R(c_norm[LA][ia] * c_norm[LB][ib] * c_norm[LC][ic] * c_norm[LD][id]);
            }
        }
        __syncthreads();
        if (active) {
            if (args.mode == MODE_EXPORT) {
                double *o = args.out + args.out_off[qi];
                for (int c = lane; c < NCART; c += TQ) o[c] = s_out[c];
            } else {
                const int n = args.n;
                const int fa = args.pr.fa[u], fb = args.pr.fb[u], fc = args.pr.fa[v], fd = args.pr.fb[v];
                const bool sab = args.pr.sa[u] == args.pr.sb[u], scd = args.pr.sa[v] == args.pr.sb[v];
                const double deg = (sab ? 1.0 : 2.0) * (scd ? 1.0 : 2.0) * (u == v ? 1.0 : 2.0);
                const int mode = args.mode;
                const double sJ = mode == MODE_RHF ? 0.5 * deg : 0.25 * deg;
                const double sK = 0.125 * deg;
                const double *D0 = args.D0, *D1 = args.D1;
                constexpr int T0 = NA * NB, T1 = T0 + NC * ND, T2 = T1 + NA * NC, T3 = T2 + NA * ND,
                              T4 = T3 + NB * NC, T5 = T4 + NB * ND;
                for (int t = lane; t < T5; t += TQ) {
                    if (t < T1) {
                        // Coulomb: J(ab) over kets or J(cd) over bras, density Dsum
                        double s = 0.0;
                        int row, col;
                        if (t < T0) {
                            const int i = t / NB, j = t % NB;
                            row = fa + i; col = fb + j;
                            for (int k = 0; k < NC; ++k)
                                for (int l = 0; l < ND; ++l) {
                                    double d = __ldg(D0 + (size_t)(fc + k) * n + fd + l);
                                    if (mode == MODE_UHF) d += __ldg(D1 + (size_t)(fc + k) * n + fd + l);
                                    s = fma((double)s_out[((i * NB + j) * NC + k) * ND + l], d, s);
                                }
                        } else {
                            const int tt = t - T0, k = tt / ND, l = tt % ND;
                            row = fc + k; col = fd + l;
                            for (int i = 0; i < NA; ++i)
                                for (int j = 0; j < NB; ++j) {
                                    double d = __ldg(D0 + (size_t)(fa + i) * n + fb + j);
                                    if (mode == MODE_UHF) d += __ldg(D1 + (size_t)(fa + i) * n + fb + j);
                                    s = fma((double)s_out[((i * NB + j) * NC + k) * ND + l], d, s);
                                }
                        }
                        s *= sJ;
                        acc_add(args.A0, (size_t)row * n + col, s, args.det, args.err);
                        if (mode == MODE_UHF) acc_add(args.A1, (size_t)row * n + col, s, args.det, args.err);
                    } else {
                        // exchange: four index pairings
                        double s0 = 0.0, s1 = 0.0;
                        int row, col;
                        const bool two = mode == MODE_UHF;
                        if (t < T2) {          // K(a,c) over (b,d)
                            const int tt = t - T1, i = tt / NC, k = tt % NC;
                            row = fa + i; col = fc + k;
                            for (int j = 0; j < NB; ++j)
                                for (int l = 0; l < ND; ++l) {
                                    const size_t di = (size_t)(fb + j) * n + fd + l;
                                    const double vv = (double)s_out[((i * NB + j) * NC + k) * ND + l];
                                    s0 = fma(vv, __ldg(D0 + di), s0);
                                    if (two) s1 = fma(vv, __ldg(D1 + di), s1);
                                }
                        } else if (t < T3) {   // K(a,d) over (b,c)
                            const int tt = t - T2, i = tt / ND, l = tt % ND;
                            row = fa + i; col = fd + l;
                            for (int j = 0; j < NB; ++j)
                                for (int k = 0; k < NC; ++k) {
                                    const size_t di = (size_t)(fb + j) * n + fc + k;
                                    const double vv = (double)s_out[((i * NB + j) * NC + k) * ND + l];
                                    s0 = fma(vv, __ldg(D0 + di), s0);
                                    if (two) s1 = fma(vv, __ldg(D1 + di), s1);
                                }
                        } else if (t < T4) {   // K(b,c) over (a,d)
                            const int tt = t - T3, j = tt / NC, k = tt % NC;
                            row = fb + j; col = fc + k;
                            for (int i = 0; i < NA; ++i)
                                for (int l = 0; l < ND; ++l) {
                                    const size_t di = (size_t)(fa + i) * n + fd + l;
                                    const double vv = (double)s_out[((i * NB + j) * NC + k) * ND + l];
                                    s0 = fma(vv, __ldg(D0 + di), s0);
                                    if (two) s1 = fma(vv, __ldg(D1 + di), s1);
                                }
                        } else {               // K(b,d) over (a,c)
                            const int tt = t - T4, j = tt / ND, l = tt % ND;
                            row = fb + j; col = fd + l;
                            for (int i = 0; i < NA; ++i)
                                for (int k = 0; k < NC; ++k) {
                                    const size_t di = (size_t)(fa + i) * n + fc + k;
                                    const double vv = (double)s_out[((i * NB + j) * NC + k) * ND + l];
                                    s0 = fma(vv, __ldg(D0 + di), s0);
                                    if (two) s1 = fma(vv, __ldg(D1 + di), s1);
                                }
                        }
                        const size_t o = (size_t)row * n + col;
                        if (mode == MODE_JK) {
                            acc_add(args.A1, o, sK * s0, args.det, args.err);
                        } else {
                            acc_add(args.A0, o, -sK * s0, args.det, args.err);
                            if (two) acc_add(args.A1, o, -sK * s1, args.det, args.err);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

template <int LA, int LB, int LC, int LD, typename R, int MINB = 1>
cudaError_t launch_smem(const EriArgs &a, cudaStream_t stream, int num_sms)
{
    using S = SmemShape<LA, LB, LC, LD, R>;
    static unsigned long long configured = 0;   // per device: the attribute is per device
    if (first_on_device(&configured)) {
        cudaError_t e = cudaFuncSetAttribute(eri_smem_kernel<LA, LB, LC, LD, R, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        // the hinted form needs the whole shared-memory carveout for its
        // MINB blocks; left to itself the driver may size the carveout for fewer
        if (e == cudaSuccess && MINB > 1)
            e = cudaFuncSetAttribute(eri_smem_kernel<LA, LB, LC, LD, R, MINB>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
    }
    static int resident[64] = {};
    long long blocks = (a.nquart + S::NTEAM - 1) / S::NTEAM;
    const long long cap = (long long)num_sms *
        resident_blocks((const void *)eri_smem_kernel<LA, LB, LC, LD, R, MINB>, S::BLK, S::SMEM, resident);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) return cudaSuccess;
    eri_smem_kernel<LA, LB, LC, LD, R, MINB><<<(unsigned)blocks, S::BLK, S::SMEM, stream>>>(a);
    return cudaGetLastError();
}

// FP64 occupancy-hinted form of the class (kernel variant 5); classes without
// one (HAS_OCC false) return cudaErrorInvalidValue and are never offered it.
template <int LA, int LB, int LC, int LD>
cudaError_t launch_smem_occ(const EriArgs &a, cudaStream_t stream, int num_sms)
{
    using S = SmemShape<LA, LB, LC, LD, double>;
    if constexpr (S::HAS_OCC)
        return launch_smem<LA, LB, LC, LD, double, S::OCC>(a, stream, num_sms);
    else
        return cudaErrorInvalidValue;
}

}  // namespace pg
