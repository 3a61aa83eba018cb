// gpath.cu -- kernels of the 'G' path (EnergyGA / EnergyGAM / EnergyGB,
// src/workproc.f90:1697-1950), whose reference solves H c = E S c with
// LAPACK's ZHEGVX(ITYPE=1, RANGE='I', IL=IU=WHICH_EIGENVALUE)
// (src/workproc.f90:1750).  Here the WHICH-th eigenvalue is found by
// Sylvester's law of inertia on the LDL^H factorisation of H - sigma S (its
// number of negative pivots is the number of eigenvalues below sigma),
// bisecting sigma until the bracket holds that eigenvalue alone, and then
// inverse iteration (GHEPIIS) at the bracket's centre, which no other
// eigenvalue is as close to.  The host side is ecg_abi.cu's energy_ga.
//   k_g_shift    F = A - sigma B on the lower triangle (the matrix the
//                LDL^H factorisation reads), diagonal dA - sigma dB
//   k_g_mirror   S's upper triangle from its lower one, unit diagonal (the
//                copy EnergyGA makes before ZHEGVX, src/workproc.f90:1743-1748)
//   k_g_inertia  negative pivots and the first non-positive one
#include "ecg_internal.h"

namespace ecg {

namespace {

__global__ void __launch_bounds__(256) k_g_shift(cd* __restrict__ F, const cd* __restrict__ A,
                                                 const cd* __restrict__ B, const double* __restrict__ dA,
                                                 const double* __restrict__ dB, int ld, int n, double sigma)
{
    const int j = blockIdx.y;
    for (int i = j + blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const size_t o = (size_t)i + (size_t)j * ld;
        cd v;
        if (i == j) {
            const double a = dA ? dA[i] : 1.0;
            const double b = B ? (dB ? dB[i] : 1.0) : 0.0;
            v = mk(a - sigma * b, 0.0);
        } else {
            v = A[o];
            if (B) {
                const cd bb = B[o];
                v = mk(v.x - sigma * bb.x, v.y - sigma * bb.y);
            }
        }
        F[o] = v;
    }
}

__global__ void __launch_bounds__(256) k_g_mirror(cd* __restrict__ S, int ld, int n)
{
    __shared__ double2 t[32][33];
    const int Ct = blockIdx.x, Rt = blockIdx.y;  // source tile: rows Ct (lower part), columns Rt
    if (Rt > Ct) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int q = ty; q < 32; q += 8) {
        const int r = Ct * 32 + tx, c = Rt * 32 + q;  // element (r, c), r >= c
        double2 v = make_double2(0.0, 0.0);
        if (r < n && c < n && r > c) {
            const cd a = S[(size_t)r + (size_t)c * ld];
            v = make_double2(a.x, -a.y);
        }
        t[q][tx] = v;
    }
    __syncthreads();
    for (int q = ty; q < 32; q += 8) {
        const int r = Rt * 32 + tx, c = Ct * 32 + q;  // destination (r, c), r <= c
        if (r < n && c < n) {
            if (r < c) {
                const double2 v = t[tx][q];
                S[(size_t)r + (size_t)c * ld] = cd{v.x, v.y};
            } else if (r == c) {
                S[(size_t)r + (size_t)c * ld] = cd{1.0, 0.0};
            }
        }
    }
}

__global__ void __launch_bounds__(1024) k_g_inertia(const cd* __restrict__ invD, int n, int* __restrict__ cnt)
{
    __shared__ int sneg[32], sfirst[32];
    int neg = 0, first = n;
    for (int i = threadIdx.x; i < n; i += 1024) {
        const double v = invD[i].x;  // 1 / d, real pivots; 0 for an exactly zero pivot
        if (v < 0.0) neg++;
        if (v <= 0.0 && i < first) first = i;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        neg += __shfl_xor_sync(0xffffffffu, neg, o);
        first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (lane == 0) {
        sneg[wp] = neg;
        sfirst[wp] = first;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, f = n;
        for (int w = 0; w < 32; w++) {
            a += sneg[w];
            f = min(f, sfirst[w]);
        }
        cnt[0] = a;
        cnt[1] = f;
    }
}

}  // namespace

int g_shift(Ctx& c, const cd* A, const cd* B, const double* dA, const double* dB, int n, double sigma)
{
    dim3 g((n + 255) / 256, n);
    if (g.x > 16) g.x = 16;
    k_g_shift<<<g, 256, 0, c.stream>>>(c.F, A, B, dA, dB, c.ld, n, sigma);
    c.launches++;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int g_mirror_s(Ctx& c, int n)
{
    const int nt = (n + 31) / 32;
    k_g_mirror<<<dim3(nt, nt), 256, 0, c.stream>>>(c.S, c.ld, n);
    c.launches++;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int g_inertia(Ctx& c, int n)
{
    k_g_inertia<<<1, 1024, 0, c.stream>>>(c.invD, n, c.gcnt);
    c.launches++;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace ecg
