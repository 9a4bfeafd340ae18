// onebody.cuh -- McMurchie-Davidson one-body integrals: overlap, kinetic,
// nuclear attraction and the distributed-positron-model potential.
#pragma once
#include <cuda_runtime.h>

namespace pg {

cudaError_t upload_onebody_constants();

// If S, T, H are non-null they are overwritten with the packed S, T and
// H = T + V (V over every centre but skipcen, oneints.c:139-234).  If Hdpm
// is non-null, Hdpm -= V_DPM (dpmints.c:121-199).  Host buffers; returns 0
// or a PATGPU_E* code.
int run_oneints(int nsh, const int *l, const int *cen, const int *off, const int *nst, const int *poff,
                const double *al, const double *co, int ncen, const double *q, const double *xyz, int skipcen,
                int n, double *S, double *T, double *H, double *Hdpm, cudaStream_t stream);

// Dipole (dip[3][no2]: x, y, z) and quadrupole (quad[6][no2]: xx, xy, xz,
// yy, yz, zz) integrals about the origin, packed, overwritten (host
// buffers; momints.c:13-188).
int run_moments(int nsh, const int *l, const int *cen, const int *off, const int *nst, const int *poff,
                const double *al, const double *co, int ncen, const double *xyz, int n, double *dip, double *quad,
                cudaStream_t stream);

// Nuclear gradient of the one-body energy terms 2 tr(P H) - 2 tr(W S)
// (H -= V_DPM when with_dpm) for the packed half density P and
// energy-weighted density W (W may be NULL: no overlap term).  grad[3 ncen]
// is overwritten (host buffer).
int run_onebody_grad(int nsh, const int *l, const int *cen, const int *off, const int *nst, const int *poff,
                     const double *al, const double *co, int ncen, const double *q, const double *xyz, int skipcen,
                     int n, const double *P, const double *W, int with_dpm, double *grad, cudaStream_t stream);

int fail(int code, const char *fmt, ...);

}  // namespace pg
