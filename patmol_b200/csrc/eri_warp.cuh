// eri_warp.cuh -- the warp-synchronous team variant of the shell-quartet
// kernel (variants 6 = FP64, 7 = FP32 arithmetic with FP64 roots, prefactors
// and J/K sums), for handles whose shell pairs have one primitive pair each
// (every uncontracted basis).  Same mathematics and digestion rule as
// eri_kernel.cuh (which see); the GPU mapping differs where the lane kernel
// loses time:
//
//   * A team of NL = nc*nd lanes (the ket components) lives inside one warp,
//     and a warp holds up to Q = 32/NL teams (fewer where their shared
//     memory would crowd the SM); every phase boundary is a
//     __syncwarp, never a block barrier, so the warps of an SM drift through
//     the phases independently and cover each other's latencies.
//   * The bra components are assembled in compile-time chunks of at most
//     MAXACC integrals and each chunk is digested at once: the integrals of
//     one chunk, not of the whole bra, are live in registers.
//   * The four exchange densities of the lane's ket component, D(b,d),
//     D(b,c), D(a,d) and D(a,c) over the bra components, are read into
//     registers once per quartet (for bras of up to 9 components), so the
//     digestion's FMAs take no shared-memory operand.
//   * 1/p, 1/q and 1/(p+q) are formed once per quartet, and each pair's
//     data is one 128-byte record (EriArgs::ppk) read with 128-bit loads.
//
// Per quartet and team: (A) pair data, the staged density blocks (component
// factors folded in) and the 2n Chebyshev series of the roots and weights;
// (B) the recursion + transfer jobs, (direction, root[, ket x-index]) per
// lane, into tables [dir][root][ket x-index][bra x-index]; (C) per bra chunk:
// assembly sum_r X Y Z, J(cd) and the exchange partials in registers, the
// chunk's J(ab) partials through shared memory and reduced across the team;
// (D) the exchange partials reduced across the team.  Contributions go
// through acc_add (fixed-point or FP64 atomics).
#pragma once
#include <type_traits>
#include "eri_kernel.cuh"

namespace pg {

// f(integral_constant<int, I>) for I = B .. E-1, unrolled at compile time.
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F &f)
{
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

template <int LA, int LB, int LC, int LD, int NDEN, typename R>
struct WarpShape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND, NCART = NAB * NCD;
    static constexpr int L12 = LA + LB, L34 = LC + LD;
    static constexpr int NR = (L12 + L34) / 2 + 1;
    static constexpr int TAB = (LA + 1) * (LB + 1), TCD = (LC + 1) * (LD + 1);
    static constexpr int TSZ = TAB * TCD;
    static constexpr int NL = NCD;                          // lanes per team
    static constexpr int NSPLIT = (LC > 0 && 3 * NR * (LC + 1) <= NL) ? LC + 1 : 1;
    static constexpr int NJOB = 3 * NR * NSPLIT;
    static constexpr int MAXACC = NDEN == 1 ? 18 : 12;
    static constexpr int NCH = (NAB + MAXACC - 1) / MAXACC;
    static constexpr int CH = (NAB + NCH - 1) / NCH;
    static constexpr bool DREG = NA + NB <= 9;              // exchange densities in registers
    // staged density blocks per set: D(ab), D(bd), D(bc), D(ad), D(ac)
    static constexpr int OBD = NAB, OBC = OBD + NB * ND, OAD = OBC + NB * NC, OAC = OAD + NA * ND;
    static constexpr int NDB = OAC + NA * NC;
    // staged density words per set: only D(ab) when the exchange densities
    // live in registers (DREG), all five blocks otherwise
    static constexpr int NDBS = DREG ? NAB : NDB;
    static constexpr int PS = 2 * NA + 2 * NB;              // exchange partials per lane and set
    // Shared-memory strides, chosen against bank conflicts.  Each lane's
    // recursion job writes one table of TSZ entries and each lane stores its
    // PS exchange partials; the lanes of a warp store at the same offset in
    // their own table (partial block) at once.  With odd strides TST and PSP
    // (in R and double words) and a team stride TEAM congruent to NL*TST
    // modulo 16 doubles, the 16 lanes of a half warp (one wavefront of 64-bit
    // accesses) hit 16 distinct bank pairs.  PSP is also congruent to TST
    // modulo 16, so one team stride serves both stores.
    static constexpr int TST = TSZ | 1;
    static constexpr int PSP = PS + (((TST - PS) % 16) + 16) % 16;
    // per-team shared memory, in doubles: roots/weights, staged densities,
    // tables (later the exchange partials), one chunk's J(ab) partials
    static constexpr int RW = 2 * NR;
    static constexpr int TABD = (3 * NR * TST * (int)sizeof(R) + 7) / 8;
    static constexpr int PART = NL > 1 ? NL * PSP * NDEN : 0;
    static constexpr int REGION = TABD > PART ? TABD : PART;
    // one chunk's J(ab) partials [CH][NL]; with a single bra chunk the tables
    // are dead once it is assembled, so the partials reuse their region
    // (WALIAS) and the team's shared memory shrinks by CH*NL words -- with
    // NDBS, enough to fit a fourth block on an SM for the (dp|xs), (dp|ds),
    // (pp|ss) and (dp|fs)-type classes
    static constexpr bool WALIAS = NL > 1 && NCH == 1 && CH * NL <= REGION;
    static constexpr int WCH = (NL > 1 && !WALIAS) ? CH * NL : 0;
    static constexpr int TEAM0 = RW + NDBS * NDEN + REGION + WCH;
    static constexpr int TEAM = sizeof(R) == 8 ? TEAM0 + (((NL * TST - TEAM0) % 16) + 16) % 16 : TEAM0;
    // teams per warp: 32/NL, fewer where the teams' shared memory would pass
    // 28 KB a warp (the large-bra classes with one or three ket lanes), so
    // that an SM still holds 8 or more warps
    static constexpr int QFIT = (28 * 1024) / (TEAM * 8);
    static constexpr int Q = (32 / NL) < (QFIT > 0 ? QFIT : 1) ? 32 / NL : (QFIT > 0 ? QFIT : 1);
    // warps per block: up to 4, within 200 KB of shared memory a block
    static constexpr int WFIT = (200 * 1024) / (TEAM * Q * 8);
    static constexpr int WARPS = WFIT >= 4 ? 4 : (WFIT > 0 ? WFIT : 1);
    static constexpr size_t SMEM = sizeof(double) * (size_t)TEAM * Q * WARPS;
    static_assert(SMEM <= 227 * 1024, "warp kernel shared memory");
    static_assert(NL <= 32, "the warp kernel needs at most 32 ket components");
};

template <int LA, int LB, int LC, int LD, int NDEN, typename R>
__global__ void __launch_bounds__(128, 4) eri_warp_kernel(const EriArgs args)
{
    using S = WarpShape<LA, LB, LC, LD, NDEN, R>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NAB = S::NAB;
    constexpr int NR = S::NR, TAB = S::TAB, TST = S::TST, NL = S::NL, Q = S::Q;
    constexpr int NCH = S::NCH, CH = S::CH, NDB = S::NDB, NDBS = S::NDBS, PSP = S::PSP;
    extern __shared__ double smem[];

    const int warp = threadIdx.x >> 5, wl = threadIdx.x & 31;
    const int team = wl / NL, lt = wl - team * NL;
    const bool in_team = team < Q;
    double *s_rw = smem + (size_t)(warp * Q + (in_team ? team : 0)) * S::TEAM;
    double *s_db = s_rw + S::RW;
    double *s_tab = s_db + NDBS * NDEN;         // tables; after the assembly, the exchange partials
    double *s_part = s_tab;
    double *s_wc = S::WALIAS ? s_tab : s_tab + S::REGION;   // one chunk's J(ab) partials [CH][NL]

    const int ic = lt / ND, id = lt - (lt / ND) * ND;
    const int ecx = c_cart[LC][ic], edx = c_cart[LD][id];
    const int tcdx = (ecx & 15) * (LD + 1) + (edx & 15);
    const int tcdy = ((ecx >> 4) & 15) * (LD + 1) + ((edx >> 4) & 15);
    const int tcdz = (ecx >> 8) * (LD + 1) + (edx >> 8);
    const double nfk = c_norm[LC][ic] * c_norm[LD][id];
    const int mode = args.mode;
    const int n = args.n;
    const long long stride = (long long)gridDim.x * S::WARPS * Q;
    const long long nq = eri_work_count(args), q0 = eri_work_first(args, nq);

    for (long long base = ((long long)blockIdx.x * S::WARPS + warp) * Q; base < nq; base += stride) {
        const long long qi = base + team;
        int u = 0, v = 0;
        const bool active = in_team && qi < nq && eri_quartet_at(args, q0 + qi, u, v);
        int fa = 0, fb = 0, fc = 0, fd = 0;
        double ppq = 1.0, p = 1.0, q = 1.0, sr = 0.0;
        double pax = 0, pay = 0, paz = 0, qcx = 0, qcy = 0, qcz = 0, pqx = 0, pqy = 0, pqz = 0;
        double abx = 0, aby = 0, abz = 0, cdx = 0, cdy = 0, cdz = 0;
        bool sab = false, scd = false;
        if (active) {
            // the packed pair records: one 128-byte line per pair (EriArgs::ppk)
            const double2 *Rb = reinterpret_cast<const double2 *>(args.ppk) + 8 * (size_t)u;
            const double2 *Rk = reinterpret_cast<const double2 *>(args.ppk) + 8 * (size_t)v;
            const double2 b0 = __ldg(Rb), b1 = __ldg(Rb + 1), b2 = __ldg(Rb + 2), b3 = __ldg(Rb + 3);
            const double2 b4 = __ldg(Rb + 4), b5 = __ldg(Rb + 5), b6 = __ldg(Rb + 6);
            const double2 k0 = __ldg(Rk), k1 = __ldg(Rk + 1), k2 = __ldg(Rk + 2), k3 = __ldg(Rk + 3);
            const double2 k4 = __ldg(Rk + 4), k5 = __ldg(Rk + 5), k6 = __ldg(Rk + 6);
            const unsigned long long fab = (unsigned long long)__double_as_longlong(b6.x);
            const unsigned long long fcd = (unsigned long long)__double_as_longlong(k6.x);
            const unsigned long long sb2 = (unsigned long long)__double_as_longlong(b6.y);
            const unsigned long long sk2 = (unsigned long long)__double_as_longlong(k6.y);
            fa = (int)(unsigned)(fab & 0xffffffffull); fb = (int)(unsigned)(fab >> 32);
            fc = (int)(unsigned)(fcd & 0xffffffffull); fd = (int)(unsigned)(fcd >> 32);
            sab = (sb2 & 0xffffffffull) == (sb2 >> 32);
            scd = (sk2 & 0xffffffffull) == (sk2 >> 32);
            abx = b4.y; aby = b5.x; abz = b5.y;
            cdx = k4.y; cdy = k5.x; cdz = k5.y;
            p = b0.x;
            q = k0.x;
            const double Px = b0.y, Py = b1.x, Pz = b1.y;
            const double Qx = k0.y, Qy = k1.x, Qz = k1.y;
            ppq = p + q;
            const double rs = rsqrt(ppq);
            // the primitive cut of twoints.c:109-111 drops the whole quartet
            if (kSR * b2.y * k2.y * rs >= args.prim_cut) {
                sr = kSR * b2.x * k2.x * rs;
                pax = Px - b3.x; pay = Py - b3.y; paz = Pz - b4.x;
                qcx = Qx - k3.x; qcy = Qy - k3.y; qcz = Qz - k4.x;
                pqx = Px - Qx; pqy = Py - Qy; pqz = Pz - Qz;
                const double T = p * q / ppq * (pqx * pqx + pqy * pqy + pqz * pqz);
                for (int f = lt; f < 2 * NR; f += NL) s_rw[f] = rys_eval(NR, f, T, c_rys, args.rys_coef, kRysDeg, true);
            }
            // stage D(ab) (every lane reads all of it), and with the exchange
            // densities kept in shared memory also D(bd), D(bc), D(ad), D(ac);
            // component factors folded in
#pragma unroll
            for (int s = 0; s < NDEN; ++s) {
                const double *D = s == 0 ? args.D0 : args.D1;
                double *db = s_db + s * NDBS;
                for (int t = lt; t < NAB; t += NL) {
                    const int ir = t / NB, icn = t - (t / NB) * NB;
                    db[t] = __ldg(D + (size_t)(fa + ir) * n + fb + icn) * c_norm[LA][ir] * c_norm[LB][icn];
                }
                if constexpr (!S::DREG) {
                    for (int t = lt + S::OBD; t < NDB; t += NL) {
                        int r0, c0, lr, lc2, ir, icn;
                        if (t < S::OBC) {
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
        const bool work = active && sr != 0.0;
        __syncwarp();
        if (work) {
            const double ippq = 1.0 / ppq, ip = 1.0 / p, iq = 1.0 / q;
            for (int j = lt; j < S::NJOB; j += NL) {
                const int cs = j / (3 * NR), jj = j - cs * (3 * NR);
                const int dim = jj / NR, r = jj - dim * NR;
                const double x = s_rw[r], w = s_rw[NR + r];
                const double f = x * ippq, B00 = 0.5 * f;
                const double B10 = (0.5 - B00 * q) * ip, B01 = (0.5 - B00 * p) * iq;
                const double pa = dim == 0 ? pax : (dim == 1 ? pay : paz);
                const double qc = dim == 0 ? qcx : (dim == 1 ? qcy : qcz);
                const double pq = dim == 0 ? pqx : (dim == 1 ? pqy : pqz);
                const double ab = dim == 0 ? abx : (dim == 1 ? aby : abz);
                const double cd = dim == 0 ? cdx : (dim == 1 ? cdy : cdz);
                R *tab = reinterpret_cast<R *>(s_tab) + (dim * NR + r) * TST;
                if constexpr (S::NSPLIT == 1) {
                    vrr_hrr<LA, LB, LC, LD, R>(tab, R(dim == 2 ? w * sr : 1.0), R(B00), R(B10), R(B01),
                                               R(pa - q * pq * f), R(qc + p * pq * f), R(ab), R(cd));
                } else {
#pragma unroll
                    for (int c0 = 0; c0 < S::NSPLIT; ++c0)
                        if (c0 == cs)
                            vrr_hrr<LA, LB, LC, LD, R>(tab, R(dim == 2 ? w * sr : 1.0), R(B00), R(B10), R(B01),
                                                       R(pa - q * pq * f), R(qc + p * pq * f), R(ab), R(cd), c0);
                }
            }
        }
        __syncwarp();

        // ------------------------------------------------------ digestion
        sab = sab && work;
        scd = scd && work;
        const double deg = (sab ? 1.0 : 2.0) * (scd ? 1.0 : 2.0) * (u == v ? 1.0 : 2.0);
        const double sJ = mode == MODE_RHF ? 0.5 * deg : 0.25 * deg;
        const double sK = 0.125 * deg;
        double Dcd = 0.0, jcd = 0.0;
        double Pac[NDEN][NA], Pad[NDEN][NA], Pbc[NDEN][NB], Pbd[NDEN][NB];
        double dbd[NDEN][S::DREG ? NB : 1], dbc[NDEN][S::DREG ? NB : 1];
        double dad[NDEN][S::DREG ? NA : 1], dac[NDEN][S::DREG ? NA : 1];
#pragma unroll
        for (int s = 0; s < NDEN; ++s) {
#pragma unroll
            for (int a = 0; a < NA; ++a) { Pac[s][a] = 0.0; Pad[s][a] = 0.0; }
#pragma unroll
            for (int b = 0; b < NB; ++b) { Pbc[s][b] = 0.0; Pbd[s][b] = 0.0; }
        }
        if (work) {
            Dcd = __ldg(args.D0 + (size_t)(fc + ic) * n + fd + id);
            if (NDEN == 2) Dcd += __ldg(args.D1 + (size_t)(fc + ic) * n + fd + id);
            Dcd *= nfk;
            if constexpr (S::DREG) {
                // this lane's exchange densities straight from the n x n
                // density (consecutive ket components read consecutive words)
                const double nd = c_norm[LD][id], nc = c_norm[LC][ic];
#pragma unroll
                for (int s = 0; s < NDEN; ++s) {
                    const double *D = s == 0 ? args.D0 : args.D1;
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        dbd[s][b] = __ldg(D + (size_t)(fb + b) * n + fd + id) * (c_norm[LB][b] * nd);
                        dbc[s][b] = __ldg(D + (size_t)(fb + b) * n + fc + ic) * (c_norm[LB][b] * nc);
                    }
#pragma unroll
                    for (int a = 0; a < NA; ++a) {
                        dad[s][a] = __ldg(D + (size_t)(fa + a) * n + fd + id) * (c_norm[LA][a] * nd);
                        dac[s][a] = __ldg(D + (size_t)(fa + a) * n + fc + ic) * (c_norm[LA][a] * nc);
                    }
                }
            }
        }
        const R *tb = reinterpret_cast<const R *>(s_tab);
        const R *X = tb + tcdx * TAB;
        const R *Y = tb + NR * TST + tcdy * TAB;
        const R *Z = tb + 2 * NR * TST + tcdz * TAB;
        auto chunk = [&](auto cst) {
            constexpr int c = decltype(cst)::value;
            constexpr int CHN = (c + 1) * CH <= NAB ? CH : NAB - c * CH;
            R acc[CH];
#pragma unroll
            for (int j = 0; j < CH; ++j) acc[j] = R(0);
            if (work) assemble<LA, LB, NR, TST, c * CH, CH>(acc, X, Y, Z);
            // the J(ab) partials below overwrite the tables (WALIAS): every
            // lane of the warp has finished its table reads first
            if constexpr (S::WALIAS) __syncwarp();
            if (work) {
#pragma unroll
                for (int j = 0; j < CHN; ++j) {
                    const int ab = c * CH + j;
                    const int ia = ab / NB, ib = ab % NB;
                    const double I = (double)acc[j];
                    double dab = s_db[ab];
                    if (NDEN == 2) dab += s_db[NDBS + ab];
                    jcd = fma(I, dab, jcd);
                    if constexpr (NL > 1) {
                        s_wc[j * NL + lt] = I * Dcd;
                    } else {
                        const double o = sJ * I * Dcd * c_norm[LA][ia] * c_norm[LB][ib];
                        const size_t idx = (size_t)(fa + ia) * n + fb + ib;
                        acc_add(args.A0, idx, o, args.det, args.err);
                        if (NDEN == 2) acc_add(args.A1, idx, o, args.det, args.err);
                    }
#pragma unroll
                    for (int s = 0; s < NDEN; ++s) {
                        if constexpr (S::DREG) {
                            Pac[s][ia] = fma(I, dbd[s][ib], Pac[s][ia]);
                            Pad[s][ia] = fma(I, dbc[s][ib], Pad[s][ia]);
                            Pbc[s][ib] = fma(I, dad[s][ia], Pbc[s][ib]);
                            Pbd[s][ib] = fma(I, dac[s][ia], Pbd[s][ib]);
                        } else {
                            const double *db = s_db + s * NDBS;
                            Pac[s][ia] = fma(I, db[S::OBD + ib * ND + id], Pac[s][ia]);
                            Pad[s][ia] = fma(I, db[S::OBC + ib * NC + ic], Pad[s][ia]);
                            Pbc[s][ib] = fma(I, db[S::OAD + ia * ND + id], Pbc[s][ib]);
                            Pbd[s][ib] = fma(I, db[S::OAC + ia * NC + ic], Pbd[s][ib]);
                        }
                    }
                }
            }
            if constexpr (NL > 1) {
                // this chunk's J(ab): sum over the team's ket components
                __syncwarp();
                if (work) {
                    for (int t = lt; t < CHN; t += NL) {
                        double sum = 0.0;
#pragma unroll 6
                        for (int k = 0; k < NL; ++k) sum += s_wc[t * NL + k];
                        const int ab = c * CH + t, ia = ab / NB, ib = ab - (ab / NB) * NB;
                        const double o = sJ * sum * c_norm[LA][ia] * c_norm[LB][ib];
                        const size_t idx = (size_t)(fa + ia) * n + fb + ib;
                        acc_add(args.A0, idx, o, args.det, args.err);
                        if (NDEN == 2) acc_add(args.A1, idx, o, args.det, args.err);
                    }
                }
                __syncwarp();
            }
        };
        static_for<0, NCH>(chunk);
        if (work) {
            // J(cd): complete in this lane
            const double o = sJ * jcd * nfk;
            const size_t idx = (size_t)(fc + ic) * n + fd + id;
            acc_add(args.A0, idx, o, args.det, args.err);
            if (NDEN == 2) acc_add(args.A1, idx, o, args.det, args.err);
        }
        if constexpr (NL == 1) {
            if (work) {
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
            }
        } else {
            // exchange partials through shared memory (the tables are dead:
            // the last chunk's barrier ordered every table read before this)
            if (work) {
#pragma unroll
                for (int s = 0; s < NDEN; ++s) {
                    double *pp = s_part + ((size_t)s * NL + lt) * PSP;
#pragma unroll
                    for (int a = 0; a < NA; ++a) { pp[a] = Pac[s][a]; pp[NA + a] = Pad[s][a]; }
#pragma unroll
                    for (int b = 0; b < NB; ++b) { pp[2 * NA + b] = Pbc[s][b]; pp[2 * NA + NB + b] = Pbd[s][b]; }
                }
            }
            __syncwarp();
            if (work) {
                // K(a,c) = sum_d Pac, K(a,d) = sum_c Pad, K(b,c) = sum_d Pbc,
                // K(b,d) = sum_c Pbd over the team's ket components (lane
                // c*ND + d holds the partials of ket component (c, d))
#pragma unroll
                for (int s = 0; s < NDEN; ++s) {
                    double *A = mode == MODE_JK ? args.A1 : (s == 0 ? args.A0 : args.A1);
                    const double sg = mode == MODE_JK ? sK : -sK;
                    const double *pp = s_part + (size_t)s * NL * PSP;
                    for (int t = lt; t < NA * NC; t += NL) {
                        const int a = t / NC, c = t - (t / NC) * NC;
                        double sum = 0.0;
#pragma unroll
                        for (int d = 0; d < ND; ++d) sum += pp[(c * ND + d) * PSP + a];
                        acc_add(A, (size_t)(fa + a) * n + fc + c, sg * c_norm[LA][a] * c_norm[LC][c] * sum, args.det,
                                args.err);
                    }
                    for (int t = lt; t < NA * ND; t += NL) {
                        const int a = t / ND, d = t - (t / ND) * ND;
                        double sum = 0.0;
#pragma unroll
                        for (int c = 0; c < NC; ++c) sum += pp[(c * ND + d) * PSP + NA + a];
                        acc_add(A, (size_t)(fa + a) * n + fd + d, sg * c_norm[LA][a] * c_norm[LD][d] * sum, args.det,
                                args.err);
                    }
                    for (int t = lt; t < NB * NC; t += NL) {
                        const int b = t / NC, c = t - (t / NC) * NC;
                        double sum = 0.0;
#pragma unroll
                        for (int d = 0; d < ND; ++d) sum += pp[(c * ND + d) * PSP + 2 * NA + b];
                        acc_add(A, (size_t)(fb + b) * n + fc + c, sg * c_norm[LB][b] * c_norm[LC][c] * sum, args.det,
                                args.err);
                    }
                    for (int t = lt; t < NB * ND; t += NL) {
                        const int b = t / ND, d = t - (t / ND) * ND;
                        double sum = 0.0;
#pragma unroll
                        for (int c = 0; c < NC; ++c) sum += pp[(c * ND + d) * PSP + 2 * NA + NB + b];
                        acc_add(A, (size_t)(fb + b) * n + fd + d, sg * c_norm[LB][b] * c_norm[LD][d] * sum, args.det,
                                args.err);
                    }
                }
            }
        }
        // the next quartet's staging and roots overwrite this team's region
        __syncwarp();
    }
}

template <int LA, int LB, int LC, int LD, int NDEN, typename R = double>
cudaError_t launch_warp(const EriArgs &a, cudaStream_t stream, int num_sms)
{
    using S = WarpShape<LA, LB, LC, LD, NDEN, R>;
    static unsigned long long configured = 0;   // per device: the attribute is per device
    if (first_on_device(&configured)) {
        cudaError_t e = cudaFuncSetAttribute(eri_warp_kernel<LA, LB, LC, LD, NDEN, R>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return e;
    }
    static int resident[64] = {};
    const long long per_block = (long long)S::Q * S::WARPS;
    long long blocks = (a.nquart + per_block - 1) / per_block;
    const long long cap = (long long)num_sms * resident_blocks((const void *)eri_warp_kernel<LA, LB, LC, LD, NDEN, R>,
                                                               32 * S::WARPS, S::SMEM, resident);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) return cudaSuccess;
    eri_warp_kernel<LA, LB, LC, LD, NDEN, R><<<(unsigned)blocks, 32 * S::WARPS, S::SMEM, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace pg
