// common.cuh -- shared device/host helpers of the patgpu library:
// Cartesian component tables in the reference's order, Rys roots from the
// generated Chebyshev tables, and the Boys function for the MD kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

#define PG_LMAX 3            // kernels are instantiated up to f shells
#define PG_NROOT_MAX 7       // (ff|ff): L = 12 -> 7 roots
#define PG_HD __host__ __device__ __forceinline__

namespace pg {

constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

#ifdef __CUDACC__
// One-time per-device set-up (kernel attributes, constant tables): true the
// first time the current device asks through this mask (bit d for device d).
inline bool first_on_device(unsigned long long *mask)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return true;
    const unsigned long long bit = 1ull << (dev & 63);
    return !(__atomic_fetch_or(mask, bit, __ATOMIC_ACQ_REL) & bit);
}

// Blocks of `func` (block threads, smem dynamic bytes) that one SM holds at
// once, from the occupancy calculator, cached per device in cache[64] (0 =
// not yet asked).  The class kernels loop grid-stride over their quartets,
// so a grid of this many blocks per SM runs as one wave: no partial last
// wave leaves SMs idle at the end of a launch.
inline int resident_blocks(const void *func, int block, size_t smem, int *cache)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    dev &= 63;
    int v = __atomic_load_n(cache + dev, __ATOMIC_ACQUIRE);
    if (v > 0) return v;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, func, block, smem) != cudaSuccess || occ < 1) occ = 1;
    __atomic_store_n(cache + dev, occ, __ATOMIC_RELEASE);
    return occ;
}
#endif

// Cartesian exponents in the order of basis.c:294-308: lx descending, then
// ly descending.  Packed as lx | ly << 4 | lz << 8 for l <= 3.
struct CartTab {
    int e[4][10];
};
constexpr CartTab make_cart_tab()
{
    CartTab t{};
    for (int l = 0; l <= 3; ++l) {
        int n = 0;
        for (int lx = l; lx >= 0; --lx)
            for (int ly = l - lx; ly >= 0; --ly) {
                t.e[l][n] = lx | (ly << 4) | ((l - lx - ly) << 8);
                ++n;
            }
    }
    return t;
}
constexpr CartTab kCart = make_cart_tab();

// host-side accessors (device code reads the same table from constant memory)
inline int cart_x(int l, int k) { return kCart.e[l][k] & 15; }
inline int cart_y(int l, int k) { return (kCart.e[l][k] >> 4) & 15; }
inline int cart_z(int l, int k) { return (kCart.e[l][k] >> 8) & 15; }

// 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!) (basis.c:309-319)
PG_HD double dfact_odd(int l)
{
    return l <= 1 ? 1.0 : (l == 2 ? 3.0 : (l == 3 ? 15.0 : (l == 4 ? 105.0 : 945.0)));
}

// ---------------------------------------------------------------- Rys
// Tables live in device global memory (coefficients) and constant memory
// (offsets, limits, large-T nodes); see rys_table.h.
struct RysConst {
    int tmax[10];
    int off[10];
    double lag_x[10][9];
    double lag_w[10][9];
};

// Evaluate function f (0..n-1: node x = t^2, n..2n-1: weight) of the
// n-root Rys rule at T.  Chebyshev series (Clenshaw) on unit intervals
// below tmax[n], generalised-Laguerre limit above.
// Coefficient layouts, per n from rc.off[n] and per interval k a block of
// 2n (deg+1) doubles: series-major, coefficient j of function f at
// f (deg+1) + j (rys_table.h as generated, interleaved = false), or
// coefficient-major at j 2n + f (interleaved = true: the copy on the
// device, where the lanes evaluating one quartet's 2n series read
// neighbouring words at every step).
PG_HD double rys_eval(int n, int f, double T, const RysConst &rc, const double *__restrict__ coef,
                      int deg, bool interleaved = false)
{
    if (!(T < (double)rc.tmax[n])) {   // also takes NaN: no table access
        if (f < n) return rc.lag_x[n][f] / T;
        return rc.lag_w[n][f - n] / sqrt(T);
    }
    int k = (int)T;
    double u = 2.0 * (T - (double)k) - 1.0;
    const size_t blk = rc.off[n] + (size_t)k * 2 * n * (deg + 1);
    const double *c = coef + blk + (interleaved ? (size_t)f : (size_t)f * (deg + 1));
    const int cs = interleaved ? 2 * n : 1;
    double b1 = 0.0, b2 = 0.0, u2 = 2.0 * u;
    for (int j = deg; j >= 1; --j) {
#ifdef __CUDA_ARCH__
        double cj = __ldg(c + j * cs);
#else
        double cj = c[j * cs];
#endif
        double t = fma(u2, b1, cj - b2);
        b2 = b1;
        b1 = t;
    }
#ifdef __CUDA_ARCH__
    double c0 = __ldg(c);
#else
    double c0 = c[0];
#endif
    return fma(u, b1, c0 - b2);
}

// The coefficient-major copy of a series-major table (see rys_eval); nmax
// functions sets, rc.off[nmax + 1] = total size.
inline void rys_interleave(const double *src, double *dst, const int *off, const int *tmax, int nmax, int deg)
{
    for (int n = 1; n <= nmax; ++n)
        for (int k = 0; k < tmax[n]; ++k) {
            const size_t blk = off[n] + (size_t)k * 2 * n * (deg + 1);
            for (int f = 0; f < 2 * n; ++f)
                for (int j = 0; j <= deg; ++j) dst[blk + (size_t)j * 2 * n + f] = src[blk + (size_t)f * (deg + 1) + j];
        }
}

// ---------------------------------------------------------------- Boys
// F_m(T), m = 0..mmax (mmax <= 16): Taylor series at mmax and downward
// recursion below T = 30; above, F_0 = sqrt(pi/T)/2 erf(sqrt T) and upward
// recursion F_{m+1} = ((2m+1) F_m - e^-T)/(2T), which is stable for T > m.
PG_HD void boys(int mmax, double T, double *F)
{
    if (T < 30.0) {
        double e = exp(-T);
        double term = 1.0 / (2 * mmax + 1), sum = term;
        for (int i = 1; i < 200; ++i) {
            term *= 2.0 * T / (2 * mmax + 2 * i + 1);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        F[mmax] = e * sum;
        for (int m = mmax - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + e) / (2 * m + 1);
    } else {
        double st = sqrt(T);
        double e = exp(-T);
        F[0] = 0.886226925452758013649 * erf(st) / st;
        for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
    }
}

}  // namespace pg
