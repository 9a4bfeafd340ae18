// eri_reg.cuh -- the register-only variant of the shell-quartet kernel, for
// the small classes whose whole integral block fits in one thread's
// registers.  Same mathematics and digestion rule as eri_kernel.cuh; here one
// thread owns one quartet from start to finish: no shared memory, no block
// barriers, no team bookkeeping.  For these classes the per-quartet set-up
// of a team, not the arithmetic, dominates.
#pragma once
#include "eri_kernel.cuh"

namespace pg {

template <int LA, int LB, int LC, int LD>
struct RegShape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND, NCART = NAB * NCD;
    static constexpr int L12 = LA + LB, L34 = LC + LD;
    static constexpr int NR = (L12 + L34) / 2 + 1;
    static constexpr int TAB = (LA + 1) * (LB + 1), TCD = (LC + 1) * (LD + 1);
    static constexpr int TSZ = TAB * TCD;
};

// One root, one direction: 2-D recursion and binomial transfer into the
// register table t[(c(LD+1)+d) TAB + a(LB+1)+b].
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void vrr_hrr_reg(double (&t)[RegShape<LA, LB, LC, LD>::TSZ], double g00, double B00,
                                            double B10, double B01, double C, double Cp, double ab, double cd)
{
    constexpr int L12 = LA + LB, L34 = LC + LD, TAB = (LA + 1) * (LB + 1);
    double G[L12 + 1][L34 + 1];
    G[0][0] = g00;
    if (L12 > 0) G[1][0] = C * g00;
#pragma unroll
    for (int i = 1; i < L12; ++i) G[i + 1][0] = i * B10 * G[i - 1][0] + C * G[i][0];
#pragma unroll
    for (int j = 0; j < L34; ++j)
#pragma unroll
        for (int i = 0; i <= L12; ++i) {
            double v = Cp * G[i][j];
            if (j > 0) v = fma(j * B01, G[i][j - 1], v);
            if (i > 0) v = fma(i * B00, G[i - 1][j], v);
            G[i][j + 1] = v;
        }
    double cdp[LD + 1], abp[LB + 1];
    cdp[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= LD; ++k) cdp[k] = cdp[k - 1] * cd;
    abp[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= LB; ++k) abp[k] = abp[k - 1] * ab;
#pragma unroll
    for (int c = 0; c <= LC; ++c)
#pragma unroll
        for (int d = 0; d <= LD; ++d) {
            double H[L12 + 1];
#pragma unroll
            for (int i = 0; i <= L12; ++i) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k <= d; ++k) s = fma(binom(d, k) * cdp[k], G[i][c + d - k], s);
                H[i] = s;
            }
#pragma unroll
            for (int a = 0; a <= LA; ++a)
#pragma unroll
                for (int b = 0; b <= LB; ++b) {
                    double s = 0.0;
#pragma unroll
                    for (int i = 0; i <= b; ++i) s = fma(binom(b, i) * abp[i], H[a + b - i], s);
                    t[(c * (LD + 1) + d) * TAB + a * (LB + 1) + b] = s;
                }
        }
}

template <int LA, int LB, int LC, int LD, int NDEN>
__global__ void __launch_bounds__(128, 4) eri_reg_kernel(const EriArgs args)
{
    using S = RegShape<LA, LB, LC, LD>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NAB = S::NAB, NCD = S::NCD;
    constexpr int NCART = S::NCART, NR = S::NR, TAB = S::TAB, TSZ = S::TSZ;
    const int n = args.n;
    const int mode = args.mode;
    const double *__restrict__ D0 = args.D0;
    const double *__restrict__ D1 = args.D1;

    const long long nq = eri_work_count(args), q0 = eri_work_first(args, nq);
    for (long long qi = (long long)blockIdx.x * blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x) {
        int u, v;
        if (!eri_quartet_at(args, q0 + qi, u, v)) continue;
        double ax, ay, az, abx, aby, abz, cx, cy, cz, cdx, cdy, cdz;
        int fa, fb, fc, fd;
        bool sab, scd;

        double I[NCART];
#pragma unroll
        for (int c = 0; c < NCART; ++c) I[c] = 0.0;

        // one primitive quartet: p, P, K, the coefficient-free prefactor of
        // the bra pair, the same of the ket pair
        auto prim = [&](double p, double Px, double Py, double Pz, double Kb, double cb, double qx, double Qx,
                        double Qy, double Qz, double Kk, double ck) {
            const double ppq = p + qx, rs = rsqrt(ppq);
            if (kSR * cb * ck * rs < args.prim_cut) return;   // twoints.c:109-111
            const double sr = kSR * Kb * Kk * rs;
            const double pax = Px - ax, pay = Py - ay, paz = Pz - az;
            const double qcx = Qx - cx, qcy = Qy - cy, qcz = Qz - cz;
            const double pqx = Px - Qx, pqy = Py - Qy, pqz = Pz - Qz;
            const double T = p * qx / ppq * (pqx * pqx + pqy * pqy + pqz * pqz);
#pragma unroll 1
            for (int r = 0; r < NR; ++r) {
                const double x = rys_eval(NR, r, T, c_rys, args.rys_coef, kRysDeg, true);
                const double w = rys_eval(NR, NR + r, T, c_rys, args.rys_coef, kRysDeg, true);
                const double f = x / ppq, B00 = 0.5 * f;
                const double B10 = (0.5 - B00 * qx) / p, B01 = (0.5 - B00 * p) / qx;
                double tx[TSZ], ty[TSZ], tz[TSZ];
                vrr_hrr_reg<LA, LB, LC, LD>(tx, 1.0, B00, B10, B01, pax - qx * pqx * f, qcx + p * pqx * f, abx, cdx);
                vrr_hrr_reg<LA, LB, LC, LD>(ty, 1.0, B00, B10, B01, pay - qx * pqy * f, qcy + p * pqy * f, aby, cdy);
                vrr_hrr_reg<LA, LB, LC, LD>(tz, w * sr, B00, B10, B01, paz - qx * pqz * f, qcz + p * pqz * f, abz,
                                            cdz);
#pragma unroll
                for (int ab = 0; ab < NAB; ++ab)
#pragma unroll
                    for (int cd = 0; cd < NCD; ++cd) {
                        const int ia = ab / NB, ib2 = ab % NB, ic = cd / ND, id = cd % ND;
                        const int ox = (cexp(LC, ic, 0) * (LD + 1) + cexp(LD, id, 0)) * TAB +
                                       cexp(LA, ia, 0) * (LB + 1) + cexp(LB, ib2, 0);
                        const int oy = (cexp(LC, ic, 1) * (LD + 1) + cexp(LD, id, 1)) * TAB +
                                       cexp(LA, ia, 1) * (LB + 1) + cexp(LB, ib2, 1);
                        const int oz = (cexp(LC, ic, 2) * (LD + 1) + cexp(LD, id, 2)) * TAB +
                                       cexp(LA, ia, 2) * (LB + 1) + cexp(LB, ib2, 2);
                        I[ab * NCD + cd] = fma(tx[ox] * ty[oy], tz[oz], I[ab * NCD + cd]);
                    }
            }
        };

        if (args.ppk) {
            // one-primitive handles: each pair is one 128-byte record
            // (EriArgs::ppk) read with seven 128-bit loads, instead of
            // fourteen scattered words of the pair and primitive arrays
            const double2 *Rb = reinterpret_cast<const double2 *>(args.ppk) + 8 * (size_t)u;
            const double2 *Rk = reinterpret_cast<const double2 *>(args.ppk) + 8 * (size_t)v;
            const double2 b0 = __ldg(Rb), b1 = __ldg(Rb + 1), b2 = __ldg(Rb + 2), b3 = __ldg(Rb + 3);
            const double2 b4 = __ldg(Rb + 4), b5 = __ldg(Rb + 5), b6 = __ldg(Rb + 6);
            const double2 k0 = __ldg(Rk), k1 = __ldg(Rk + 1), k2 = __ldg(Rk + 2), k3 = __ldg(Rk + 3);
            const double2 k4 = __ldg(Rk + 4), k5 = __ldg(Rk + 5), k6 = __ldg(Rk + 6);
            ax = b3.x; ay = b3.y; az = b4.x; abx = b4.y; aby = b5.x; abz = b5.y;
            cx = k3.x; cy = k3.y; cz = k4.x; cdx = k4.y; cdy = k5.x; cdz = k5.y;
            const unsigned long long fab = (unsigned long long)__double_as_longlong(b6.x);
            const unsigned long long fcd = (unsigned long long)__double_as_longlong(k6.x);
            const unsigned long long sb2 = (unsigned long long)__double_as_longlong(b6.y);
            const unsigned long long sk2 = (unsigned long long)__double_as_longlong(k6.y);
            fa = (int)(unsigned)(fab & 0xffffffffull); fb = (int)(unsigned)(fab >> 32);
            fc = (int)(unsigned)(fcd & 0xffffffffull); fd = (int)(unsigned)(fcd >> 32);
            sab = (sb2 & 0xffffffffull) == (sb2 >> 32);
            scd = (sk2 & 0xffffffffull) == (sk2 >> 32);
            prim(b0.x, b0.y, b1.x, b1.y, b2.x, b2.y, k0.x, k0.y, k1.x, k1.y, k2.x, k2.y);
        } else {
            ax = args.pr.ax[u]; ay = args.pr.ay[u]; az = args.pr.az[u];
            abx = args.pr.abx[u]; aby = args.pr.aby[u]; abz = args.pr.abz[u];
            cx = args.pr.ax[v]; cy = args.pr.ay[v]; cz = args.pr.az[v];
            cdx = args.pr.abx[v]; cdy = args.pr.aby[v]; cdz = args.pr.abz[v];
            fa = args.pr.fa[u]; fb = args.pr.fb[u]; fc = args.pr.fa[v]; fd = args.pr.fb[v];
            sab = args.pr.sa[u] == args.pr.sb[u];
            scd = args.pr.sa[v] == args.pr.sb[v];
            const int npb = args.pr.pnum[u], npk = args.pr.pnum[v];
            const int pb0 = args.pr.pstart[u], pk0 = args.pr.pstart[v];
            for (int ib = pb0; ib < pb0 + npb; ++ib)
                for (int ik = pk0; ik < pk0 + npk; ++ik)
                    prim(args.pp.p[ib], args.pp.px[ib], args.pp.py[ib], args.pp.pz[ib], args.pp.K[ib],
                         args.pp.cut[ib], args.pp.p[ik], args.pp.px[ik], args.pp.py[ik], args.pp.pz[ik],
                         args.pp.K[ik], args.pp.cut[ik]);
        }

        if (mode == MODE_EXPORT) {
            double *o = args.out + args.out_off[qi];
#pragma unroll
            for (int ab = 0; ab < NAB; ++ab)
#pragma unroll
                for (int cd = 0; cd < NCD; ++cd) {
                    const double val = I[ab * NCD + cd] * c_norm[LA][ab / NB] * c_norm[LB][ab % NB] *
                                       c_norm[LC][cd / ND] * c_norm[LD][cd % ND];
                    o[args.swap ? (size_t)cd * NAB + ab : (size_t)ab * NCD + cd] = val;
                }
            continue;
        }

        // component factors folded into the integrals once
#pragma unroll
        for (int ab = 0; ab < NAB; ++ab)
#pragma unroll
            for (int cd = 0; cd < NCD; ++cd)
                I[ab * NCD + cd] *= c_norm[LA][ab / NB] * c_norm[LB][ab % NB] * c_norm[LC][cd / ND] *
                                    c_norm[LD][cd % ND];

        const double deg = (sab ? 1.0 : 2.0) * (scd ? 1.0 : 2.0) * (u == v ? 1.0 : 2.0);
        const double sJ = mode == MODE_RHF ? 0.5 * deg : 0.25 * deg;
        const double sK = 0.125 * deg;
        auto dsum = [&](int r, int c) {
            double d = __ldg(D0 + (size_t)r * n + c);
            if (NDEN == 2) d += __ldg(D1 + (size_t)r * n + c);
            return d;
        };
        // Coulomb: J(ab) over the ket, J(cd) over the bra
#pragma unroll
        for (int ab = 0; ab < NAB; ++ab) {
            double s = 0.0;
#pragma unroll
            for (int cd = 0; cd < NCD; ++cd) s = fma(I[ab * NCD + cd], dsum(fc + cd / ND, fd + cd % ND), s);
            const size_t o = (size_t)(fa + ab / NB) * n + fb + ab % NB;
            acc_add(args.A0, o, sJ * s, args.det, args.err);
            if (NDEN == 2) acc_add(args.A1, o, sJ * s, args.det, args.err);
        }
#pragma unroll
        for (int cd = 0; cd < NCD; ++cd) {
            double s = 0.0;
#pragma unroll
            for (int ab = 0; ab < NAB; ++ab) s = fma(I[ab * NCD + cd], dsum(fa + ab / NB, fb + ab % NB), s);
            const size_t o = (size_t)(fc + cd / ND) * n + fd + cd % ND;
            acc_add(args.A0, o, sJ * s, args.det, args.err);
            if (NDEN == 2) acc_add(args.A1, o, sJ * s, args.det, args.err);
        }
        // exchange: K(a,c) over (b,d), K(a,d) over (b,c), K(b,c) over (a,d), K(b,d) over (a,c)
#pragma unroll
        for (int s = 0; s < NDEN; ++s) {
            const double *__restrict__ D = s == 0 ? D0 : D1;
            double *A = mode == MODE_JK ? args.A1 : (s == 0 ? args.A0 : args.A1);
            const double sg = mode == MODE_JK ? sK : -sK;
#pragma unroll
            for (int a = 0; a < NA; ++a) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    double k = 0.0;
#pragma unroll
                    for (int b = 0; b < NB; ++b)
#pragma unroll
                        for (int d = 0; d < ND; ++d)
                            k = fma(I[(a * NB + b) * NCD + c * ND + d], __ldg(D + (size_t)(fb + b) * n + fd + d), k);
                    acc_add(A, (size_t)(fa + a) * n + fc + c, sg * k, args.det, args.err);
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    double k = 0.0;
#pragma unroll
                    for (int b = 0; b < NB; ++b)
#pragma unroll
                        for (int c = 0; c < NC; ++c)
                            k = fma(I[(a * NB + b) * NCD + c * ND + d], __ldg(D + (size_t)(fb + b) * n + fc + c), k);
                    acc_add(A, (size_t)(fa + a) * n + fd + d, sg * k, args.det, args.err);
                }
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    double k = 0.0;
#pragma unroll
                    for (int a = 0; a < NA; ++a)
#pragma unroll
                        for (int d = 0; d < ND; ++d)
                            k = fma(I[(a * NB + b) * NCD + c * ND + d], __ldg(D + (size_t)(fa + a) * n + fd + d), k);
                    acc_add(A, (size_t)(fb + b) * n + fc + c, sg * k, args.det, args.err);
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    double k = 0.0;
#pragma unroll
                    for (int a = 0; a < NA; ++a)
#pragma unroll
                        for (int c = 0; c < NC; ++c)
                            k = fma(I[(a * NB + b) * NCD + c * ND + d], __ldg(D + (size_t)(fa + a) * n + fc + c), k);
                    acc_add(A, (size_t)(fb + b) * n + fd + d, sg * k, args.det, args.err);
                }
            }
        }
    }
}

template <int LA, int LB, int LC, int LD, int NDEN>
cudaError_t launch_reg(const EriArgs &a, cudaStream_t stream, int num_sms)
{
    static int resident[64] = {};
    long long blocks = (a.nquart + 127) / 128;
    const long long cap =
        (long long)num_sms * resident_blocks((const void *)eri_reg_kernel<LA, LB, LC, LD, NDEN>, 128, 0, resident);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) return cudaSuccess;
    eri_reg_kernel<LA, LB, LC, LD, NDEN><<<(unsigned)blocks, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace pg
