// zmma.cuh -- complex FP64 tile products on the tensor cores
// (mma.sync.aligned.m8n8k4.f64; tcgen05 has no f64 kind) and cp.async
// staging helpers, shared by the batched-candidate kernels.
//
// Shared-memory operand layouts, double2 = (re, im):
//   A tile  As[k * LDA + m]   k-major, LDA % 8 == 2
//   B tile  Bs[n * LDB + k]   n-major, LDB % 8 == 4
// so that the fragment loads of one quarter-warp (lanes g = lane/4 in
// {0,1}, t = lane%4) touch eight distinct 16-byte bank groups.
// A complex multiply-accumulate is four real mma: Re += Ar Br - Ai Bi,
// Im += Ar Bi + Ai Br (the minus folded into a negated fragment).
#pragma once
#include <cuda_runtime.h>

namespace ecg {

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Accumulators of one warp: MT x NT tiles of 8 x 8; thread (g, t) holds
// C(g, 2t + e), e = 0, 1, of every tile.
template <int MT, int NT>
struct ZAcc {
    double r[MT][NT][2];
    double i[MT][NT][2];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int a = 0; a < MT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) r[a][b][0] = r[a][b][1] = i[a][b][0] = i[a][b][1] = 0.0;
    }
};

// acc += op(A)(wm.., kk..kk+3) * B(kk..kk+3, wn..); op = conj when CONJA.
template <int MT, int NT, int LDA, int LDB, bool CONJA>
__device__ __forceinline__ void zmma_k4(ZAcc<MT, NT>& acc, const double2* __restrict__ As,
                                        const double2* __restrict__ Bs, int wm, int wn, int kk, int lane)
{
    const int g = lane >> 2, t = lane & 3;
    double ar[MT], ai[MT], an[MT], br[NT], bi[NT];
#pragma unroll
    for (int mt = 0; mt < MT; mt++) {
        const double2 a = As[(kk + t) * LDA + wm + mt * 8 + g];
        ar[mt] = a.x;
        ai[mt] = CONJA ? -a.y : a.y;
        an[mt] = -ai[mt];
    }
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
        const double2 b = Bs[(wn + nt * 8 + g) * LDB + kk + t];
        br[nt] = b.x;
        bi[nt] = b.y;
    }
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
            dmma(acc.r[mt][nt][0], acc.r[mt][nt][1], ar[mt], br[nt]);
            dmma(acc.r[mt][nt][0], acc.r[mt][nt][1], an[mt], bi[nt]);
            dmma(acc.i[mt][nt][0], acc.i[mt][nt][1], ar[mt], bi[nt]);
            dmma(acc.i[mt][nt][0], acc.i[mt][nt][1], ai[mt], br[nt]);
        }
}

// 16-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros
// (the source is then not read).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace ecg
